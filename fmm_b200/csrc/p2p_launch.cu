// The streamed mixed P2P's launches, in a translation unit of their own: its kernels do
// not depend on the expansion order, so they are compiled once, not once per order.
#include "p2p_x2.cuh"

namespace fmmb {

namespace {
template <int W, int KS>
void launch_wk(const P2pStArgs& a, unsigned grid, cudaStream_t s) {
    if (a.m == 1)
        p2p_st_kernel<true, W, true, KS><<<grid, 32 * W, 0, s>>>(a);
    else
        p2p_st_kernel<true, W, false, KS><<<grid, 32 * W, 0, s>>>(a);
}

template <int W>
void launch_w(const P2pStArgs& a, int ks, unsigned grid, cudaStream_t s) {
    switch (ks) {
        case 1: launch_wk<W, 1>(a, grid, s); break;
        case 2: launch_wk<W, 2>(a, grid, s); break;
        case 4: launch_wk<W, 4>(a, grid, s); break;
        case 8: launch_wk<W, 8>(a, grid, s); break;
        default: launch_wk<W, 0>(a, grid, s);
    }
}
}  // namespace

void launch_p2p_st(const P2pStArgs& a, int warps, int ks, unsigned grid, cudaStream_t s) {
    if (warps == 1)
        launch_w<1>(a, ks, grid, s);
    else if (warps == 2)
        launch_w<2>(a, ks, grid, s);
    else
        launch_w<4>(a, ks, grid, s);
}

}  // namespace fmmb
