// Kernels compiled with -use_fast_math: the arithmetic of the reference's _C_benchmarking and
// _C_stereo modules (setup.py:63-99 of the reference builds those with -O3 -use_fast_math).
#define FHTGS_FLAVOR fast
// bulk-copy staging of the preprocess attributes (see launch_preprocess_t)
constexpr bool kStagedPreprocess = true;
#include "fhtgs_kernels.cuh"
namespace fhtgs {
const KernelSet& kernels_fast() { return fast::kernel_set(); }
}  // namespace fhtgs
