# Compiles oracle/ref_layout_probe.cpp against the reference's own layout header (a header-only,
# dependency-free file of the reference tree) into oracle/_ref/ref_layout and writes its JSON to
# tests/golden/ref_layout.json. Run from the repository root with the reference tree's location:
# make -f oracle/ref_layout.mk REFERENCE=<path to the reference tree> (or CAELIX_REFERENCE set in the
# environment).
REFERENCE ?= $(CAELIX_REFERENCE)
ifeq ($(REFERENCE),)
$(error set REFERENCE (or CAELIX_REFERENCE) to the reference tree)
endif

tests/golden/ref_layout.json: oracle/_ref/ref_layout
	oracle/_ref/ref_layout > $@

oracle/_ref/ref_layout: oracle/ref_layout_probe.cpp $(REFERENCE)/lib/src/light/light_tree_layout.h
	@mkdir -p oracle/_ref
	g++ -std=c++20 -O0 -I$(REFERENCE)/lib/src oracle/ref_layout_probe.cpp -o $@
