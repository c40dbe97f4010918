# Compiles oracle/ref_layout_probe.cpp against the reference's own layout header (a header-only,
# dependency-free file of the reference tree) into oracle/_ref/ref_layout and writes its JSON to
# tests/golden/ref_layout.json. Run from the repository root: make -f oracle/ref_layout.mk
REFERENCE ?= /root/reference

tests/golden/ref_layout.json: oracle/_ref/ref_layout
	oracle/_ref/ref_layout > $@

oracle/_ref/ref_layout: oracle/ref_layout_probe.cpp $(REFERENCE)/lib/src/light/light_tree_layout.h
	@mkdir -p oracle/_ref
	g++ -std=c++20 -O0 -I$(REFERENCE)/lib/src oracle/ref_layout_probe.cpp -o $@
