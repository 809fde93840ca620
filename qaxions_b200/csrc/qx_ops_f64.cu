// Plain FP64 (complex128) instantiation of the pass launchers.
#include "qx_ops_impl.cuh"
namespace qx {
template struct Ops<double>;
}  // namespace qx
