// Host launchers of the box-8-colour block ILU(0) kernels (ewg_box8.cuh).
#include "ewg_box8.cuh"

namespace ewg {

namespace {

int b8_grid(ewg_ctx* ctx, const void* kernel) {
    int g = grid_size_for(ctx, kernel, kSolBlock);
    const int64_t need = (ctx->P.Nb + kSolBlock - 1) / kSolBlock;
    return (int)(need < g ? (need > 0 ? need : 1) : g);
}

// sweeps: one block per tile of 32 superblocks, at most the resident blocks of one wave
int b8_sweep_grid(ewg_ctx* ctx, const void* kernel) {
    int g = grid_size_for(ctx, kernel, kB8Block);
    const int64_t need = (ctx->P.Nb + 31) / 32;
    return (int)(need < g ? (need > 0 ? need : 1) : g);
}

template <typename T, int C>
void factor_colour(ewg_ctx* ctx, const T* A8, T* Dinv8, T* L8, T* E8, int* bad) {
    auto kfn = k_b8_factor<T, C>;
    EWG_LAUNCH(ctx, K_B8_FACTOR, kfn, b8_grid(ctx, (const void*)kfn), kSolBlock, ctx->P, A8, Dinv8, L8, E8, bad);
}

template <typename T, int C>
void forward_colour(ewg_ctx* ctx, const T* L8, const typename V2T<T>::type* d, typename V2T<T>::type* y,
                    const int* status) {
    auto kfn = k_b8_forward<T, T, C>;
    EWG_LAUNCH_PDL(ctx, K_B8_FORWARD, kfn, b8_sweep_grid(ctx, (const void*)kfn), kB8Block, ctx->P, L8, d, y, status);
}

template <typename T, int C>
void backward_colour(ewg_ctx* ctx, const T* A8, const T* Dinv8, const typename V2T<T>::type* w,
                     typename V2T<T>::type* y, const int* status, double relax) {
    auto kfn = k_b8_backward<T, T, C>;
    EWG_LAUNCH_PDL(ctx, K_B8_BACKWARD, kfn, b8_sweep_grid(ctx, (const void*)kfn), kB8Block, ctx->P, A8, Dinv8, w, y,
                   status, relax);
}

}  // namespace

template <typename TI, typename TO>
void b8_matrix_from_split(ewg_ctx* ctx, int nPlanes, const TI* in, TO* out) {
    auto kfn = k_b8_matrix_from_split<TI, TO>;
    EWG_LAUNCH(ctx, K_B8_LAYOUT, kfn, grid_size_for(ctx, (const void*)kfn, kSolBlock), kSolBlock, ctx->P, nPlanes,
               in, out);
}

template <typename TI, typename TO, bool TOB8>
void b8_vector(ewg_ctx* ctx, const typename V2T<TI>::type* in, typename V2T<TO>::type* out) {
    auto kfn = k_b8_vector<TI, TO, TOB8>;
    EWG_LAUNCH(ctx, K_B8_LAYOUT, kfn, grid_size_for(ctx, (const void*)kfn, kSolBlock), kSolBlock, ctx->P, in, out);
}

template <typename T>
void b8_factor(ewg_ctx* ctx, const T* A8, T* Dinv8, T* L8, T* E8, int* bad) {
    factor_colour<T, 0>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 1>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 2>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 3>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 4>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 5>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 6>(ctx, A8, Dinv8, L8, E8, bad);
    factor_colour<T, 7>(ctx, A8, Dinv8, L8, E8, bad);
}

template <typename T>
void b8_apply(ewg_ctx* ctx, const T* A8, const T* Dinv8, const T* L8, double relax,
              const typename V2T<T>::type* d, typename V2T<T>::type* w, typename V2T<T>::type* y, const int* status) {
    forward_colour<T, 0>(ctx, L8, d, w, status);
    forward_colour<T, 1>(ctx, L8, d, w, status);
    forward_colour<T, 2>(ctx, L8, d, w, status);
    forward_colour<T, 3>(ctx, L8, d, w, status);
    forward_colour<T, 4>(ctx, L8, d, w, status);
    forward_colour<T, 5>(ctx, L8, d, w, status);
    forward_colour<T, 6>(ctx, L8, d, w, status);
    forward_colour<T, 7>(ctx, L8, d, w, status);
    backward_colour<T, 7>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 6>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 5>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 4>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 3>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 2>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 1>(ctx, A8, Dinv8, w, y, status, relax);
    backward_colour<T, 0>(ctx, A8, Dinv8, w, y, status, relax);
}

template void b8_matrix_from_split<double, double>(ewg_ctx*, int, const double*, double*);
template void b8_matrix_from_split<float, float>(ewg_ctx*, int, const float*, float*);
template void b8_vector<double, double, true>(ewg_ctx*, const double2*, double2*);
template void b8_vector<double, double, false>(ewg_ctx*, const double2*, double2*);
template void b8_vector<double, float, true>(ewg_ctx*, const double2*, float2*);
template void b8_vector<float, float, false>(ewg_ctx*, const float2*, float2*);
template void b8_factor<double>(ewg_ctx*, const double*, double*, double*, double*, int*);
template void b8_factor<float>(ewg_ctx*, const float*, float*, float*, float*, int*);
template void b8_apply<double>(ewg_ctx*, const double*, const double*, const double*, double, const double2*, double2*,
                               double2*, const int*);
template void b8_apply<float>(ewg_ctx*, const float*, const float*, const float*, double, const float2*, float2*,
                              float2*, const int*);

}  // namespace ewg
