// Golden vectors of the reference's radix sort test (tests/light_tree_test.cpp:1460-1515 of the
// reference): std::mt19937(3), n in {1, 2, 1000, 100000}, 30-bit keys with many duplicates
// (one in three a multiple of 0x00FFFFF below 64 * 0x00FFFFF), values = input index, expected
// = std::sort of the (key, index) pairs. Writes, per n, the input keys and the sorted pairs as
// little-endian u32 to <out_dir>/sort_n<n>_{keys,sorted_keys,sorted_values}.bin.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <random>
#include <string>
#include <utility>
#include <vector>

static void write(const std::string& path, const std::vector<uint32_t>& v)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(v.data(), 4, v.size(), f);
    std::fclose(f);
}

int main(int argc, char** argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    std::mt19937 rng(3);
    for (const uint32_t n : {1u, 2u, 1000u, 100000u})
    {
        std::vector<uint32_t> keys(n), sk(n), sv(n);
        std::vector<std::pair<uint32_t, uint32_t>> expected(n);
        for (uint32_t i = 0; i < n; ++i)
        {
            uint32_t key;
            if (rng() % 3 == 0)
                key = (rng() % 64) * 0x00FFFFFu;
            else
                key = rng() & 0x3FFFFFFFu;
            keys[i] = key;
            expected[i] = {key, i};
        }
        std::sort(expected.begin(), expected.end());
        for (uint32_t i = 0; i < n; ++i)
        {
            sk[i] = expected[i].first;
            sv[i] = expected[i].second;
        }
        const std::string base = dir + "/sort_n" + std::to_string(n);
        write(base + "_keys.bin", keys);
        write(base + "_sorted_keys.bin", sk);
        write(base + "_sorted_values.bin", sv);
    }
    return 0;
}
