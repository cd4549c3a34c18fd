// Host check of the split-FP16 field scales (ens::fp16_field_scale): prints, for each
// case of field maxima given on the command line as 4 floats, the four scales and their
// inverses.  Built and run by tests/test_fp16_scales.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../rbf-fd-swe_b200/csrc/ens_operands.cuh"

int main(int argc, char** argv) {
    if (argc != 5) return 2;
    unsigned bits[4];
    for (int f = 0; f < 4; ++f) {
        const float v = std::strtof(argv[1 + f], nullptr);
        std::memcpy(&bits[f], &v, sizeof(v));
    }
    for (int f = 0; f < 4; ++f)
        std::printf("%a %a\n", swe::ens::fp16_field_scale(bits, f, false), swe::ens::fp16_field_scale(bits, f, true));
    return 0;
}
