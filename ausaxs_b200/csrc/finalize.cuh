// Device-side manager post-processing (see finalize.cu).
#pragma once
#include "common.cuh"

namespace ausaxs_b200 {

enum FFKind : int32_t { kKindAvg = 2, kKindExplicit = 3, kKindGrid = 4 };

// Compact FP64 row layout of a form-factor histogram (T dense atom types):
//   [0, T*T)           aa (t_i, t_j), factor and self terms applied
//   [T*T, T*T+T)       ax (t)  : [ff][exv]
//   T*T+T              xx      : [exv][exv]
//   [T*T+T+1, T*T+2T+1) aw (t)
//   T*T+2T+1           wx      : aw[exv]
//   T*T+2T+2           ww
__host__ __device__ inline int ff_rows(int T) { return T * T + 2 * T + 3; }

struct FinalizeFF {
    int32_t kind;
    int32_t T;
    int32_t nb;  // bins allocated (stride of every array)
    int32_t n_a, n_w, n_x;
    const int32_t* type_count;  // [T] atoms per dense type
    const int32_t* ff_to_type;  // [15] form_factor_t -> dense type or -1
    const unsigned long long* cnt_aa;
    const unsigned long long* cnt_aw;
    const unsigned long long* cnt_ww;
    const unsigned long long* cnt_ax;
    const unsigned long long* cnt_wx;
    const unsigned long long* cnt_xx;
    const unsigned long long* ds_aa;
    const unsigned long long* ds_aw;
    const unsigned long long* ds_ww;
    const unsigned long long* ds_ax;
    const unsigned long long* ds_wx;
    const unsigned long long* ds_xx;
    double z_exv;
    double bin_width;
    float c, scale;
    int32_t weighted;
    int32_t* max_bin;  // device, preset to 10
    double* H;         // [ff_rows(T)][nb]
    double* tot;       // [nb]
    double* d_axis;    // [nb]
    double* d_axis_ax; // [nb] (grid)
    double* d_axis_xx; // [nb] (grid)
};

// Simple / weighted histogram: rows {aa, aw, ww} of weighted counts.
struct FinalizeMT {
    int32_t nb;
    const unsigned long long *c_aa, *c_aw, *c_ww;
    const unsigned long long *ds_aa, *ds_aw, *ds_ww;
    const long long *w_aa, *w_aw, *w_ww;
    const float* wscale;
    const double* self_aa;  // sum float(w*w) over atoms
    const double* self_ww;
    double bin_width;
    float c, scale;
    int32_t weighted;
    int32_t* max_bin;
    double* H;  // [3][nb]
    double* tot;
    double* d_axis;
};

void ff_finalize_launch(const FinalizeFF& F, cudaStream_t s);
// the same for n structures at once (device array of descriptors; max_nb >= every nb)
void ff_finalize_batch_launch(const FinalizeFF* Fs_dev, int n, int max_nb, cudaStream_t s);
void ff_expand_launch(const FinalizeFF& F, double* aa_out, double* aw_out, int nb_hint, cudaStream_t s);
void mt_finalize_launch(const FinalizeMT& F, cudaStream_t s);
void weight_scale_launch(const float4* a, int na, const float4* b, int nb, float* wscale, cudaStream_t s);
void weight_square_sum_launch(const float4* p, int n, double* out, cudaStream_t s);

}  // namespace ausaxs_b200
