"""Recipe: compile the reference's own device header on the CPU, as a pin for the oracle.

The reference keeps its key maps (d_u32/d_u64) and built-in operators (Maximum, Minimum,
EqualTo, ...) in built_in.h (built_in.h:14-150,430-458).  That header is plain C++ once
``__device__`` is defined away, so this recipe compiles it, where it lies in the reference
tree, together with a small driver written here, into ``oracle/_ref/ref_probe`` and runs it
on a fixed list of edge values.  The printed results become tests/golden/builtin_h_probe.json
(via tests/golden/make_golden.py), which the CPU tests compare the oracle against.

The whole reference library is built by oracle/build_ref.py (its kernels then run on a GPU
through NVRTC); this probe needs no GPU.  Test infrastructure only.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
sys.path.insert(0, os.path.dirname(HERE))
from oracle.build_ref import ref_root  # noqa: E402  (the reference tree this recipe reads)

REF_ROOT = ref_root()

DRIVER = r"""
#include <cstdint>
#include <cstddef>
#include <cstdio>
#include <cstring>
#define DEVICE_ONLY
#define __device__
#include "built_in.h"

static const uint32_t F32_BITS[] = {
    0x00000000u, 0x80000000u, 0x3F800000u, 0xBF800000u, 0x40000000u, 0xC0000000u,
    0x7F800000u, 0xFF800000u, 0x7FC00000u, 0xFFC00000u, 0x7F800001u, 0xFF800001u,
    0x00000001u, 0x80000001u, 0x7F7FFFFFu, 0xFF7FFFFFu, 0x7FFFFFFFu, 0xFFFFFFFFu};
static const uint64_t F64_BITS[] = {
    0x0000000000000000ull, 0x8000000000000000ull, 0x3FF0000000000000ull, 0xBFF0000000000000ull,
    0x7FF0000000000000ull, 0xFFF0000000000000ull, 0x7FF8000000000000ull, 0xFFF8000000000000ull,
    0x0000000000000001ull, 0x8000000000000001ull, 0x7FEFFFFFFFFFFFFFull, 0xFFEFFFFFFFFFFFFFull};
static const int64_t INTS[] = {0, 1, -1, 127, -128, 255, 32767, -32768, 65535, 2147483647,
                               -2147483647 - 1, 4294967295LL, 9223372036854775807LL,
                               -9223372036854775807LL - 1};

int main() {
    printf("{\n\"f32\": [");
    for (size_t i = 0; i < sizeof(F32_BITS) / 4; i++) {
        float f; memcpy(&f, &F32_BITS[i], 4);
        printf("%s[%u, %u]", i ? ", " : "", F32_BITS[i], d_u32<float>(f));
    }
    printf("],\n\"f64\": [");
    for (size_t i = 0; i < sizeof(F64_BITS) / 8; i++) {
        double d; memcpy(&d, &F64_BITS[i], 8);
        printf("%s[\"%llu\", \"%llu\"]", i ? ", " : "", (unsigned long long)F64_BITS[i],
               (unsigned long long)d_u64<double>(d));
    }
    printf("],\n\"ints\": [");
    for (size_t i = 0; i < sizeof(INTS) / 8; i++) {
        int64_t v = INTS[i];
        printf("%s[\"%lld\", %u, %u, %u, %u, %u, %u, \"%llu\", \"%llu\"]", i ? ", " : "", (long long)v,
               d_u32<int8_t>((int8_t)v), d_u32<uint8_t>((uint8_t)v), d_u32<int16_t>((int16_t)v),
               d_u32<uint16_t>((uint16_t)v), d_u32<int32_t>((int32_t)v), d_u32<uint32_t>((uint32_t)v),
               (unsigned long long)d_u64<int64_t>(v), (unsigned long long)d_u64<uint64_t>((uint64_t)v));
    }
    // Maximum / Minimum on float pairs with NaN and signed zeros (built_in.h:23-39)
    printf("],\n\"maxmin_f32\": [");
    const float vals[] = {1.0f, -1.0f, 0.0f, -0.0f, __builtin_nanf(""), 2.5f};
    int first = 1;
    for (float x : vals) for (float y : vals) {
        Maximum mx; Minimum mn; float a = mx(x, y), b = mn(x, y);
        uint32_t ax, bx, xx, yx; memcpy(&ax, &a, 4); memcpy(&bx, &b, 4); memcpy(&xx, &x, 4); memcpy(&yx, &y, 4);
        printf("%s[%u, %u, %u, %u]", first ? "" : ", ", xx, yx, ax, bx); first = 0;
    }
    printf("]\n}\n");
    return 0;
}
"""


def build_and_run():
    """Returns the parsed probe output, or None when the reference tree is absent."""
    header = os.path.join(REF_ROOT, "built_in.h")
    if not os.path.exists(header):
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    src = os.path.join(OUT_DIR, "ref_probe.cpp")
    exe = os.path.join(OUT_DIR, "ref_probe")
    with open(src, "w") as f:
        f.write(DRIVER)
    subprocess.check_call(["g++", "-std=c++17", "-O0", "-I", REF_ROOT, src, "-o", exe])
    out = subprocess.check_output([exe]).decode()
    return json.loads(out)


if __name__ == "__main__":
    res = build_and_run()
    if res is None:
        print("reference tree not present; nothing built")
        sys.exit(0)
    json.dump(res, sys.stdout, indent=1)
