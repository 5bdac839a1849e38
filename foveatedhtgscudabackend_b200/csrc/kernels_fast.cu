// Kernels compiled with -use_fast_math: the arithmetic of the reference's _C_benchmarking and
// _C_stereo modules (setup.py:63-99 of the reference builds those with -O3 -use_fast_math).
#define FHTGS_FLAVOR fast
#include "fhtgs_kernels.cuh"
namespace fhtgs {
const KernelSet& kernels_fast() { return fast::kernel_set(); }
}  // namespace fhtgs
