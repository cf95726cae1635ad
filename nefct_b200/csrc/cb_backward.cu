// Instantiations of the cone-beam transpose (backprojection) kernels (one direction per
// translation unit so the two compile in parallel).
#include "cb_kernels.cuh"

namespace nefct {

template <typename T>
cudaError_t cb_launch_backward(CBParams<T> &p, int na, int nb, int nvc, uint32_t flags, cudaStream_t s, bool colwarp)
{
    if constexpr (std::is_same<T, float>::value) {
        if (colwarp) return cb_launch_colwarp<false>(p, na, nb, nvc, s);
    }
    return cb_launch<T, false>(p, na, nb, nvc, flags, s);
}

template cudaError_t cb_launch_backward<float>(CBParams<float> &, int, int, int, uint32_t, cudaStream_t, bool);
template cudaError_t cb_launch_backward<double>(CBParams<double> &, int, int, int, uint32_t, cudaStream_t, bool);

}  // namespace nefct
