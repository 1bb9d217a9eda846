// Debye transform, FP64 per-q reduction and profile assembly (the K5 stage).
//
// For every q: sinqd[r] = sum_b H[r][b] sinc(q d_{g(r)}[b]) and
//   aa = sum F(ta,tb) sinqd_aa,   ax = sum 2 crho cx F(ta,exv) sinqd_ax,   xx = (cx crho)^2 F(x,x) sinqd_xx,
//   aw = sum 2 cw F(ta,w) sinqd_aw, wx = 2 crho cx cw F(x,w) sinqd_wx,     ww = cw^2 F(w,w) sinqd_ww,
//   I  = aa - ax + aw + xx - wx + ww,
// with Debye-Waller factors, as CompositeDistanceHistogramFFAvgBase::debye_transform
// (source/core/hist/intensity_calculator/CompositeDistanceHistogramFFAvgBase.cpp:57-76, 333-374,
// 427-558) and CompositeDistanceHistogramFFGrid (CompositeDistanceHistogramFFGrid.cpp:37-119), or
// I = exp(-q^2) sum_b (aa + cw aw + cw^2 ww) sinc for the Simple histogram (DistanceHistogram.cpp:54-87).
//
// When a tensor-core contraction (debye_x.cu, exact integer accumulation; debye_tc.cu, split BF16)
// has produced sinqd for all q, this kernel adds up its error bound per q and re-evaluates in FP64
// only the q values whose bound exceeds the tolerance: that is where cancellation between bins (and
// between profiles) bites, typically the high-q WAXS tail.
#include "debye.cuh"

namespace ausaxs_b200 {

namespace {

__constant__ FormFactor5 c_ff[kNff] = {
    {{1, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, 0},  // EXCLUDED_VOLUME (b set in ff_raw)
    {{0.456221, 3.219608, 0.812773, 2.666928, 1.380927}, {21.503498, 13.397134, 34.547137, 5.826620, 0.412902}, 0.463202},  // WATER = OH_alc
    {{0.489918, 0.262003, 0.196767, 0.049879, 0}, {20.6593, 7.74039, 49.5519, 2.20159, 0}, 0.001305},  // H
    {{2.657506, 1.078079, 1.490909, -4.241070, 0.713791}, {14.780758, 0.776775, 42.086843, -0.000294, 0.239535}, 4.297983},  // C
    {{2.909530, 0.485267, 1.516151, 0.206905, 1.541626}, {13.933084, 23.221524, 41.990403, 4.974183, 0.679266}, 0.337670},  // CH
    {{3.275723, 0.870037, 1.534606, 0.395078, 1.544562}, {13.408502, 23.785175, 41.922444, 5.019072, 0.724439}, 0.377096},  // CH2
    {{3.681341, 1.228691, 1.549320, 0.574033, 1.554377}, {13.026207, 24.131974, 41.869426, 4.984373, 0.765769}, 0.409294},  // CH3
    {{11.893780, 3.277479, 1.858092, 0.858927, 0.912985}, {0.000158, 10.232723, 30.344690, 0.656065, 0.217287}, -11.804902},  // N
    {{1.650531, 0.429639, 2.144736, 1.851894, 1.408921}, {10.603730, 6.987283, 29.939901, 10.573859, 0.611678}, 0.510589},  // NH
    {{1.904157, 1.942536, 2.435585, 0.730512, 1.379728}, {10.803702, 10.792421, 29.610479, 6.847755, 0.709687}, 0.603738},  // NH2
    {{1.882162, 1.933200, 2.465843, 0.927311, 1.190889}, {10.975157, 10.956008, 29.208572, 6.663555, 0.843650}, 0.597322},  // NH3
    {{2.960427, 2.508818, 0.637853, 0.722838, 1.142756}, {14.182259, 5.936858, 0.112726, 34.958481, 0.390240}, 0.027014},  // O
    {{6.362157, 5.154568, 1.473732, 1.635073, 1.209372}, {1.514347, 22.092528, 0.061373, 55.445176, 0.646925}, 0.154722},  // S
    {{0.570042, 6.337416, 1.641643, 5.398549, 1.527982}, {11.447986, 1.197657, 55.401032, 22.420955, 2.356552}, 1.523944},  // SH
    {{7.188004, 6.638454, 0.454180, 1.929593, 1.523654}, {0.956221, 15.339877, 15.339862, 39.043824, 0.062409}, 0.265954},  // OTHER (Ar)
};

constexpr double kPi = 3.14159265358979323846;
constexpr double kRhoWater = 0.334;        // e / A^3 (include/core/constants/Constants.h:114)
constexpr double kAvgRadius = 1.62;        // A (Constants.h:90)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kCB = 128;                       // bins per staged chunk
constexpr int kRG = 32;                        // rows per group of register accumulators
constexpr int kMaxRows = 264;

// Excluded volume (A^3) per form_factor_t for explicit excluded volume: the reference's default set
// constants::exv::MinimumFluctuation_implicit_H (include/core/form_factor/ExvTable.h:67-81), in the
// order of ExvFormFactorSet::get (ExvFormFactor.h:53-72); OTHER is the argon sphere 4 pi/3 1.88^3
// (ExvTable.h:135, vdwTable.h:13).  Entry 0 (the excluded volume itself) is never used.
__constant__ double c_exv_volume[kNff] = {0.0,    20.911, 0.0,    12.352, 11.640, 34.583, 41.851, 0.027,
                                          2.181,  20.562, 20.722, 14.238, 15.413, 28.529,
                                          4.0 * 3.14159265358979323846 / 3.0 * 1.88 * 1.88 * 1.88};

__device__ double ff_raw(int t, double q) {
    const FormFactor5& f = c_ff[t];
    const double s_to_q = 1.0 / (4 * 4 * kPi * kPi);
    double sum = 0;
    for (int i = 0; i < 5; ++i) {
        double b = t == kExv ? (i == 0 ? kAvgRadius * kAvgRadius / 2 : 0.0) : f.b[i] * s_to_q;
        sum += f.a[i] * exp(-b * q * q);
    }
    return sum + f.c;
}

// VectorDebyeTable::initialize (source/core/table/VectorDebyeTable.cpp:24-40)
__device__ __forceinline__ double sinc64(double x) {
    if (x < 1e-3) {
        double x2 = x * x;
        return 1 - x2 * (1.0 / 6) + x2 * x2 * (1.0 / 120);
    }
    return sin(x) / x;
}

struct QFactors {
    double f[kNff];  // raw atomic form factors at q
    double fx;       // excluded-volume form factor at q (FFAvg, FFGrid)
    double xe[kNff]; // per-type excluded-volume form factors at q (FFExplicit)
    double e;        // FFExplicit exv_factor(q) = cx^3 exp(-(r^2/4)(cx^2 - 1) q^2), r = 1.62 A
    double ba, bx;   // Debye-Waller factors
    double eq2;      // exp(-q^2)
};

// The profiles one histogram row contributes to and with which coefficient (<= 3 terms); profile
// indices {aa, ax, aw, xx, wx, ww} = 0..5.  Simple rows carry the cw powers of I here (the profiles
// themselves do not), so sum_terms sign(p) * cf is the row's coefficient in I.
struct RowTerms {
    int n;
    int p[3];
    double cf[3];
    double in_I;  // coefficient of the row's sinc sum in I
};

__device__ RowTerms row_terms(const DebyeArgs& A, const RowDesc& r, const QFactors& F) {
    RowTerms t{};
    auto add = [&](int p, double c) {
        t.p[t.n] = p;
        t.cf[t.n] = c;
        ++t.n;
        t.in_I += (p == 1 || p == 4) ? -c : c;
    };
    switch (r.kind) {
        case kRowAA: add(0, (F.f[r.ta] * F.f[r.tb]) * F.ba * F.ba); break;
        case kRowAX: add(1, 2 * A.crho * A.cx * (F.f[r.ta] * F.fx) * F.ba * F.bx); break;
        case kRowXX: add(3, (A.cx * A.crho) * (A.cx * A.crho) * (F.fx * F.fx) * F.bx * F.bx); break;
        case kRowAW: add(2, 2 * A.cw * (F.f[r.ta] * F.f[kWater]) * F.ba); break;
        case kRowWX: add(4, 2 * A.crho * A.cx * A.cw * (F.fx * F.f[kWater]) * F.bx); break;
        case kRowWW: add(5, A.cw * A.cw * (F.f[kWater] * F.f[kWater])); break;
        case kRowSAA: add(0, F.eq2); break;
        case kRowSAW:
            add(2, F.eq2);
            t.in_I *= A.cw;
            break;
        case kRowSWW:
            add(5, F.eq2);
            t.in_I *= A.cw * A.cw;
            break;
        case kRowEAA:
            add(0, (F.f[r.ta] * F.f[r.tb]) * F.ba * F.ba);
            add(1, A.crho * F.e * (F.f[r.ta] * F.xe[r.tb] + F.f[r.tb] * F.xe[r.ta]) * F.ba * F.bx);
            add(3, (F.e * A.crho) * (F.e * A.crho) * (F.xe[r.ta] * F.xe[r.tb]) * F.bx * F.bx);
            break;
        case kRowEAW:
            add(2, 2 * A.cw * (F.f[r.ta] * F.f[kWater]) * F.ba);
            add(4, A.crho * F.e * A.cw * (F.f[kWater] * F.xe[r.ta] + F.f[r.ta] * F.xe[kWater]) * F.bx);
            break;
        default: break;
    }
    return t;
}

// Factor j (0..31) of q: the 15 raw form factors, the 15 per-type excluded-volume form factors, then
// the exv factor e and the average / grid excluded-volume form factor, then the Debye-Waller factors
// and exp(-q^2).
__device__ void q_factor(const DebyeArgs& A, double q, int j, QFactors& F) {
    if (j < kNff) {
        F.f[j] = ff_raw(j, q);
    } else if (j < 2 * kNff) {
        // ExvFormFactor(V).evaluate(q) = V rho_w exp(-V^(2/3)/(4 pi) q^2) (ExvFormFactor.h:20-33)
        const double v = c_exv_volume[j - kNff];
        F.xe[j - kNff] = v * kRhoWater * exp(-(pow(v, 2.0 / 3) / (4 * kPi)) * q * q);
    } else if (j == 2 * kNff) {
        const double rm2 = kAvgRadius * kAvgRadius / 4;  // exv_factor (CompositeDistanceHistogramFFExplicitBase.cpp:54-57)
        F.e = pow(A.cx, 3) * exp(-rm2 * (pow(A.cx, 2) - 1) * q * q);
        if (A.exv_model == 1) {
            const double e = pow(A.grid_volume, 2.0 / 3) / (4 * kPi);  // ExvFormFactor (ExvFormFactor.h:20-33)
            F.fx = A.grid_volume * kRhoWater * exp(-e * q * q);
        } else {
            F.fx = ff_raw(kExv, q);
        }
    } else {
        F.ba = (A.dw_atomic != 0 || A.dw_exv != 0) ? exp(-q * q * A.dw_atomic * A.dw_atomic * 0.5) : 1.0;
        F.bx = (A.dw_atomic != 0 || A.dw_exv != 0) ? exp(-q * q * A.dw_exv * A.dw_exv * 0.5) : 1.0;
        F.eq2 = exp(-q * q);
    }
}

// The per-q factor table of transforms that share q, the parameters and the excluded-volume model
// (every structure of a batch): one thread per (q, factor)
__global__ void debye_qfactors_kernel(DebyeArgs A, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nq * 32) return;
    QFactors& F = reinterpret_cast<QFactors*>(out)[i >> 5];
    q_factor(A, A.q[i >> 5], i & 31, F);
}

// q values per CTA by the transform's q count: 4 up to 256 q, 8 up to 1,024, 16 beyond.  The
// decomposition depends on nq alone, so a structure's I(q) has the same bits alone or in a batch.
constexpr int debye_qt(int nq) { return nq <= 256 ? 4 : (nq <= 1024 ? 8 : 16); }

// Layout of a CTA of QT q values: thread (warp w, lane l) owns q value l % QT and bin phase
// w * (32 / QT) + l / QT of the CTA's 256 / QT phases; a phase holds 128 QT / 256 bins of each chunk.
// Shared memory: per-q factors, the staged H chunk (reused as the cross-warp reduction buffer), the
// staged axis chunk, the row sums [QT][R] and the rows' distance-axis groups.
template <int QT>
struct QTile {
    static constexpr int kSubs = 32 / QT;
    static constexpr int kPhases = kThreads / QT;
    static constexpr int kBinsPerThread = kCB / kPhases;
    static constexpr size_t kOffRed = ((sizeof(QFactors) * QT + 15) / 16) * 16;
    static constexpr size_t kOffH = kOffRed;
    static constexpr size_t kOffAx = kOffH + sizeof(double) * kRG * kCB;
    static constexpr size_t kOffAcc = kOffAx + sizeof(double) * kCB;
    static constexpr size_t smem(int R) { return kOffAcc + sizeof(double) * QT * R + sizeof(int) * R; }
    static_assert(kWarps * kRG * QT <= kRG * kCB, "the reduction buffer must fit in the H chunk");
    static_assert(kBinsPerThread * kPhases == kCB, "a chunk must split evenly into phases");
};

// One CTA evaluates QT consecutive q values of one transform.  Each thread evaluates sinc(q d_b) for
// its q value and the bins of its phase in each 128-bin chunk once and adds H[r][b] sinc into one
// register accumulator per row (rows in groups of 32).  A (row, q) sum is therefore one serial sum per
// phase, in bin order, the phases of a warp added by shuffles and then the warps in order.
template <int QT>
__device__ void debye_qtile(const DebyeArgs& A, const int q0, unsigned char* smem) {
    using T = QTile<QT>;
    const int nqt = min(QT, A.nq - q0);
    if (nqt <= 0) return;
    const int R = A.R;
    const int mb = *A.max_bin;
    QFactors* s_F = reinterpret_cast<QFactors*>(smem);
    double* s_red = reinterpret_cast<double*>(smem + T::kOffRed);  // [kWarps][kRG][QT]
    double* s_h = reinterpret_cast<double*>(smem + T::kOffH);      // [kRG][kCB]
    double* s_ax = reinterpret_cast<double*>(smem + T::kOffAx);    // [kCB]
    double* s_acc = reinterpret_cast<double*>(smem + T::kOffAcc);  // [QT][R]
    int* s_grp = reinterpret_cast<int*>(smem + T::kOffAcc + sizeof(double) * QT * R);
    __shared__ int s_fp64[QT];
    __shared__ int s_groups;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // per-q factors: from the shared table, or 32 per q value, one per thread (a handful of exp each)
    if (A.qf) {
        constexpr int kWords = sizeof(QFactors) / sizeof(double);
        for (int i = tid; i < nqt * kWords; i += kThreads)
            reinterpret_cast<double*>(s_F)[i] = A.qf[static_cast<size_t>(q0) * kWords + i];
    } else {
        for (int i = tid; i < nqt * 32; i += kThreads) q_factor(A, A.q[q0 + (i >> 5)], i & 31, s_F[i >> 5]);
    }
    for (int qq = tid; qq < nqt; qq += kThreads) {
        s_fp64[qq] = 1;
        if (A.tc_err_est) A.tc_err_est[q0 + qq] = INFINITY;  // overwritten below when tensor-core values exist
    }
    if (tid == 0) s_groups = 1;
    for (int i = tid; i < QT * R; i += kThreads) s_acc[i] = 0;
    __syncthreads();
    for (int r = tid; r < R; r += kThreads) {
        const int g = A.rows[r].group;
        s_grp[r] = g;
        if (g > 0) atomicMax(&s_groups, g + 1);
    }

    // With tensor-core values: keep a q unless its estimated error is above tolerance.
    if (A.sinqd_tc && !(A.tc_error && *A.tc_error)) {
        // Error bound of the tensor-core values, per row: c_rel * sum_b |H||S| + c_abs * sum_b |H|.
        //  * c_rel, operand representation: H to FP32 (2^-24), FP32 sinc value (sinf 2 ulp, the
        //    division 2^-24), the BF16 products dropped by the split (< 2^-25), the main+correction
        //    sum and the FP32 partial (2^-24 each): < 2^-21 in total;
        //  * c_rel, accumulation: at most one rounding of the main accumulator per 16-bin K step
        //    (truncation allowed: 2^-23 of a magnitude no larger than twice the bound), the
        //    correction accumulator's terms are 2^-8 smaller;
        //  * c_abs: the FP32 argument q*d carries 3 roundings, i.e. |dx| <= 3 * 2^-24 x, and
        //    |d sinc/dx| <= 2/x, so |d sinc| <= 1.5 * 2^-22 for every x;
        //  * 10 % slack for the FP32 bound and row sums themselves.
        const int per = debye_tc_split_bins(mb, A.tc_splits);
        const double c_rel = (0x1p-21 + (per / 16 + 1) * 0x1p-22) * 1.1;
        const double c_abs = 0x1p-21 * 1.1;
        const size_t plane = static_cast<size_t>(R) * A.nq;
        for (int qq = warp; qq < nqt; qq += kWarps) {
            const int k = q0 + qq;
            double I = 0, err = 0;
            for (int r = lane; r < R; r += 32) {
                const double cf = row_terms(A, A.rows[r], s_F[qq]).in_I;
                double v = 0, bnd = 0, ha = 0;
                for (int z = 0; z < A.tc_splits; ++z) {
                    v += A.sinqd_tc[z * plane + static_cast<size_t>(r) * A.nq + k];
                    bnd += A.bound_tc[z * plane + static_cast<size_t>(r) * A.nq + k];
                    ha += A.habs_tc[static_cast<size_t>(z) * R + r];
                }
                s_acc[qq * R + r] = v;
                I += cf * v;
                err += fabs(cf) * (c_rel * bnd + c_abs * ha);
            }
            for (int o = 16; o > 0; o >>= 1) {
                I += __shfl_xor_sync(0xffffffffu, I, o);
                err += __shfl_xor_sync(0xffffffffu, err, o);
            }
            if (lane == 0) {
                bool ok = err <= A.tolerance * fabs(I);
                s_fp64[qq] = ok ? 0 : 1;
                if (!ok && A.fp64_columns) atomicAdd(A.fp64_columns, 1);
                if (A.tc_err_est) A.tc_err_est[k] = fabs(I) > 0 ? err / fabs(I) : INFINITY;
            }
        }
    } else if (A.x_v && !(A.tc_error && *A.tc_error)) {
        // Exact-accumulation tensor-core values (debye_x.cu): per row and split the digit and dropped-
        // pair error is at most x_e1 * Csum(q) + x_e0, Csum(q) = sum_{k,b} |C_k(b, q)| over the table;
        // the Taylor truncation adds x_ctr q^K sum |H|.  5 % slack for the FP64 sums of the bound.
        const size_t plane = static_cast<size_t>(R) * A.nq;
        for (int qq = warp; qq < nqt; qq += kWarps) {
            const int k = q0 + qq;
            double cs = 0;
            for (int c = lane; c < A.x_nch; c += 32) cs += A.x_cpart[static_cast<size_t>(c) * A.x_nqp + k];
            for (int o = 16; o > 0; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
            const double qv = A.q[k];
            double qK = 1;
            for (int j = 0; j < A.x_K; ++j) qK *= qv;
            const double trunc = A.x_ctr * qK;
            double I = 0, err = 0;
            for (int r = lane; r < R; r += 32) {
                const double cf = row_terms(A, A.rows[r], s_F[qq]).in_I;
                double v = 0, e = 0, ha = 0;
                for (int z = 0; z < A.x_splits; ++z) {
                    v += A.x_v[z * plane + static_cast<size_t>(r) * A.nq + k];
                    e += A.x_e1[static_cast<size_t>(z) * R + r] * cs + A.x_e0[static_cast<size_t>(z) * R + r];
                    ha += A.x_habs[static_cast<size_t>(z) * R + r];
                }
                s_acc[qq * R + r] = v;
                I += cf * v;
                err += fabs(cf) * (e + trunc * ha) * 1.05;
            }
            for (int o = 16; o > 0; o >>= 1) {
                I += __shfl_xor_sync(0xffffffffu, I, o);
                err += __shfl_xor_sync(0xffffffffu, err, o);
            }
            if (lane == 0) {
                bool ok = err <= A.tolerance * fabs(I);
                s_fp64[qq] = ok ? 0 : 1;
                if (!ok && A.fp64_columns) atomicAdd(A.fp64_columns, 1);
                if (A.tc_err_est) A.tc_err_est[k] = fabs(I) > 0 ? err / fabs(I) : INFINITY;
            }
        }
    }
    __syncthreads();

    int any = 0;
    for (int qq = 0; qq < nqt; ++qq) any |= s_fp64[qq];
    if (any) {
        const int qi = lane % QT, phase = warp * T::kSubs + lane / QT;
        const bool qon = qi < nqt && s_fp64[qi] != 0;
        const double q = qi < nqt ? A.q[q0 + qi] : 0.0;
        const int groups = s_groups;
        for (int rg0 = 0; rg0 < R; rg0 += kRG) {
            const int rn = min(kRG, R - rg0);
            double acc[kRG];
#pragma unroll
            for (int i = 0; i < kRG; ++i) acc[i] = 0;
            for (int g = 0; g < groups; ++g) {
                const double* axis = g == 0 ? A.axis0 : (g == 1 ? A.axis1 : A.axis2);
                for (int c0 = 0; c0 < mb; c0 += kCB) {
                    const int cn = min(kCB, mb - c0);
                    // the chunk's rows of H and axis values, coalesced, zero past the last bin
                    __syncthreads();
                    for (int i = tid; i < rn * kCB; i += kThreads) {
                        const int r = i / kCB, t = i - r * kCB;
                        s_h[i] = t < cn ? A.H[static_cast<size_t>(rg0 + r) * A.nb + c0 + t] : 0.0;
                    }
                    for (int t = tid; t < kCB; t += kThreads) s_ax[t] = t < cn ? axis[c0 + t] : 0.0;
                    __syncthreads();
                    double sv[T::kBinsPerThread];
#pragma unroll
                    for (int k = 0; k < T::kBinsPerThread; ++k) {
                        const int t = phase + k * T::kPhases;
                        sv[k] = (qon && t < cn) ? sinc64(q * s_ax[t]) : 0.0;
                    }
#pragma unroll
                    for (int i = 0; i < kRG; ++i) {
                        if (i < rn && s_grp[rg0 + i] == g) {
                            const double* h = s_h + i * kCB + phase;
                            double a = acc[i];
#pragma unroll
                            for (int k = 0; k < T::kBinsPerThread; ++k) a += h[k * T::kPhases] * sv[k];
                            acc[i] = a;
                        }
                    }
                }
            }
            // the two phases of a warp by a shuffle, then the warps in order
            __syncthreads();  // every thread is done with the staged chunk the buffer overlays
#pragma unroll
            for (int i = 0; i < kRG; ++i) {
                double v = acc[i];
#pragma unroll
                for (int o = QT; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane < QT && i < rn) s_red[(warp * kRG + i) * QT + qi] = v;
            }
            __syncthreads();
            for (int i = tid; i < rn * QT; i += kThreads) {
                const int r = i / QT, qq = i - r * QT;
                if (qq < nqt && s_fp64[qq]) {
                    double v = 0;
                    for (int w = 0; w < kWarps; ++w) v += s_red[(w * kRG + r) * QT + qq];
                    s_acc[qq * R + rg0 + r] = v;
                }
            }
            __syncthreads();
        }
    }

    for (int qq = warp; qq < nqt; qq += kWarps) {
        const int k = q0 + qq;
        double prof[6] = {0, 0, 0, 0, 0, 0};
        for (int r = lane; r < R; r += 32) {
            const RowTerms t = row_terms(A, A.rows[r], s_F[qq]);
            for (int k2 = 0; k2 < t.n; ++k2) prof[t.p[k2]] += t.cf[k2] * s_acc[qq * R + r];
        }
        for (int p = 0; p < 6; ++p)
            for (int o = 16; o > 0; o >>= 1) prof[p] += __shfl_xor_sync(0xffffffffu, prof[p], o);
        if (lane == 0) {
            double I;
            if (A.rows[0].kind >= kRowSAA && A.rows[0].kind <= kRowSWW) {
                I = prof[0] + A.cw * prof[2] + A.cw * A.cw * prof[5];
            } else {
                I = 0;
                I += prof[0];
                I -= prof[1];
                I += prof[2];
                I += prof[3];
                I -= prof[4];
                I += prof[5];
            }
            if (A.overflow && *A.overflow) I = __longlong_as_double(0x7ff8000000000000ll);
            A.Iq[k] = I;
            if (A.profiles)
                for (int p = 0; p < 6; ++p) A.profiles[static_cast<size_t>(p) * A.nq + k] = prof[p];
        }
    }
}

template <int QT>
__global__ void __launch_bounds__(kThreads, 2) debye_kernel(DebyeArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    debye_qtile<QT>(A, blockIdx.x * QT, smem);
}
// batched: blockIdx.y selects the structure
template <int QT>
__global__ void __launch_bounds__(kThreads, 2) debye_batch_kernel(const DebyeArgs* As) {
    extern __shared__ __align__(16) unsigned char smem[];
    debye_qtile<QT>(As[blockIdx.y], blockIdx.x * QT, smem);
}

template <int QT>
bool debye_configure_qt() {
    const int bytes = static_cast<int>(QTile<QT>::smem(kMaxRows));
    return cudaFuncSetAttribute(debye_kernel<QT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess &&
           cudaFuncSetAttribute(debye_batch_kernel<QT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
}
bool debye_configure() {
    static bool done = false;
    if (!done) done = debye_configure_qt<4>() && debye_configure_qt<8>() && debye_configure_qt<16>();
    return done;
}

}  // namespace

size_t debye_qfactors_doubles(int nq) { return static_cast<size_t>(nq) * (sizeof(QFactors) / sizeof(double)); }

void debye_qfactors_launch(const DebyeArgs& A, double* out, cudaStream_t s) {
    if (A.nq <= 0) return;
    debye_qfactors_kernel<<<(A.nq * 32 + 255) / 256, 256, 0, s>>>(A, out);
}

// (a failed configuration shows as the launch's own error, which the callers check)
void debye_fp64_launch(const DebyeArgs& A, cudaStream_t s) {
    debye_configure();
    switch (debye_qt(A.nq)) {
        case 4: debye_kernel<4><<<(A.nq + 3) / 4, kThreads, QTile<4>::smem(A.R), s>>>(A); break;
        case 8: debye_kernel<8><<<(A.nq + 7) / 8, kThreads, QTile<8>::smem(A.R), s>>>(A); break;
        default: debye_kernel<16><<<(A.nq + 15) / 16, kThreads, QTile<16>::smem(A.R), s>>>(A); break;
    }
}
void debye_fp64_batch_launch(const DebyeArgs* As_dev, int n, int nq, int max_R, cudaStream_t s) {
    debye_configure();
    switch (debye_qt(nq)) {
        case 4: debye_batch_kernel<4><<<dim3((nq + 3) / 4, n), kThreads, QTile<4>::smem(max_R), s>>>(As_dev); break;
        case 8: debye_batch_kernel<8><<<dim3((nq + 7) / 8, n), kThreads, QTile<8>::smem(max_R), s>>>(As_dev); break;
        default:
            debye_batch_kernel<16><<<dim3((nq + 15) / 16, n), kThreads, QTile<16>::smem(max_R), s>>>(As_dev);
            break;
    }
}

}  // namespace ausaxs_b200
