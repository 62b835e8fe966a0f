"""Writes the compile-time sys_params header the reference's sampler is built
against in oracle/_ref (same names and layout as the reference's generator,
system_parameters.cpp:9-66; values at full precision).  Part of the refmc
recipe of oracle/Makefile: python ref_sys_params.py N m exponent out.h."""
import math
import sys


def main(argv):
    N, m, expo = int(argv[0]), int(argv[1]), int(argv[2])
    out = argv[3]
    # capacity bounds for dL <= 7 (dsf adds the dL = 0 state): at most 12
    # states per call, 4 distinct parts, degree 7
    max_degree, max_parts, max_dim, multiplet, max_l = 7, 4, 16, 5, 15
    rcl = math.sqrt(2.0 * m * N)
    lines = [
        "#ifndef SYSPARAMS_H", "#define SYSPARAMS_H", "", "namespace sys_params {",
        f"    __device__ constexpr int particlesNumber = {N};",
        f"    __device__ constexpr int inverseFilling = {m};", "",
        f"    __device__ constexpr int confinementExponent = {expo};",
        "    __device__ constexpr float confinementStrength = 1.0;", "",
        f"    __device__ constexpr float RCl = {rcl!r};",
        f"    __device__ constexpr float DCl = {2 * rcl!r};",
        f"    __device__ constexpr float RCl_reciprocal = {1 / rcl!r};",
        f"    __device__ constexpr float R0_reciprocal = {2 / rcl!r};", "",
        f"    __device__ constexpr int ansatzExtendedMaxDegree = {max_degree + 1};",
        f"    __device__ constexpr int ansatzMaxPartitionSize = {max_parts};",
        f"    __device__ constexpr int ansatzSubspaceDimension = {max_dim};", "",
        f"    __device__ constexpr int ansatzMultipletSize = {multiplet};", "",
        f"    __device__ constexpr int ansatzMaxAngularMomentum = {max_l};",
        f"    __device__ constexpr int angularMomentumCutoff = {m * (N - 1) + max_l};", "",
        "}", "", "#endif", ""]
    with open(out, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main(sys.argv[1:])
