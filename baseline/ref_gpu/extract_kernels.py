"""Writes the reference's own CUDA kernel source to a build file.

The reference keeps its GPU kernels as two C++ raw string literals in
Gpu.hpp: kCudaPrelude (the CUDA spelling of its portability macros) and
kGpuKernelBody (the kernels), which its CUDA backend compiles at run time
with NVRTC (Cuda.hpp:198-257).  This script copies those two strings,
unchanged, from the reference tree into a .cu file of the build directory
(never into the repository) and appends an #include of this directory's
launch.inc, so that nvcc compiles the reference's kernels ahead of time for
sm_100a.

    python extract_kernels.py <reference>/Gpu.hpp <build>/ref_kernels.cu
"""
import re
import sys


def raw_string(text: str, name: str) -> str:
    m = re.search(r'static const char\*\s+' + name + r'\s*=\s*R"CLC\((.*?)\)CLC";', text, re.S)
    if not m:
        sys.exit(f"{name} not found")
    return m.group(1)


def main():
    src, out = sys.argv[1], sys.argv[2]
    text = open(src, encoding="utf-8-sig").read()
    with open(out, "w") as f:
        f.write("// generated from the reference's Gpu.hpp (kCudaPrelude + kGpuKernelBody); do not edit\n")
        f.write("#include <cstdint>\n")
        f.write(raw_string(text, "kCudaPrelude"))
        f.write(raw_string(text, "kGpuKernelBody"))
        f.write('\n#include "launch.inc"\n')


if __name__ == "__main__":
    main()
