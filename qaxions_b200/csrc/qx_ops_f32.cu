// Fused FP32 (complex64) instantiation of the pass launchers.
#include "qx_ops_impl.cuh"
namespace qx {
bool supported_n(int N) { return N == 4 || N == 8 || N == 16 || N == 32 || N == 64 || N == 96 || N == 128 || N == 256 || N == 512; }
template struct Ops<float>;
}  // namespace qx
