// Kernels compiled without -use_fast_math: the IEEE arithmetic of the reference's _C module.
#define FHTGS_FLAVOR ieee
// bulk-copy staging of the preprocess attributes (see launch_preprocess_t)
constexpr bool kStagedPreprocess = false;
#include "fhtgs_kernels.cuh"
namespace fhtgs {
const KernelSet& kernels_ieee() { return ieee::kernel_set(); }
}  // namespace fhtgs
