// hist::distance_calculator::SimpleCalculator<weighted_bins = true> on the device
// (include/core/hist/distance_calculator/SimpleCalculator.h:94-330): weighted self and cross jobs with
// an integer scaling factor, accumulated into results keyed by merge id.  SymmetryManagerMT
// (source/core/hist/histogram_manager/SymmetryManagerMT.cpp:37-136) issues its work this way: a
// body's self-distances once with scaling 1 + copies, and one representative of each class of
// equivalent copy pairs with the class size as scaling.
//
// Every job of one run goes into the same persistent pair launches (PairJob::mult carries the
// scaling), each result has its own integer accumulators, and one finalisation kernel turns them
// into the reference's WeightedDistribution1D entries: per bin the weight sum, the count and the
// distance sum, each 2 * scaling times the pair's contribution, plus the self diagonal
// scaling * sum(float(w*w)) in bin 0 (its count: that value truncated to unsigned, per job).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "engine.cuh"
#include "finalize.cuh"
#include "guard.cuh"
#include "pairhist.cuh"

namespace ausaxs_b200 {
namespace {

struct CalcSlot {
    unsigned long long* cnt;
    unsigned long long* ds;
    long long* ws;
    double diag_value;  // sum over the slot's self jobs of scaling * sum(float(w*w))
    double diag_count;  // sum over them of that value truncated to unsigned
    double* out;        // [3][nb]: value, count, distance sum
};

__device__ __forceinline__ double unbiased_weights(const long long* w, const unsigned long long* n, int b, double inv) {
    const unsigned long long raw = static_cast<unsigned long long>(w[b]) - n[b] * (1ull << 30);
    return static_cast<double>(static_cast<long long>(raw)) * inv;
}

// grid.y = slot; the nb accumulated bins (every later bin is zero)
__global__ void calc_finalize_kernel(const CalcSlot* slots, int nb, const float* wscale, float c, float scale) {
    const CalcSlot S = slots[blockIdx.y];
    const double inv = 1.0 / static_cast<double>(*wscale);
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const unsigned long long cnt = S.cnt[b];
        double v = 2.0 * unbiased_weights(S.ws, S.cnt, b, inv);
        double n = 2.0 * static_cast<double>(cnt);
        double d = 0;
        if (cnt) {
            // sum of the pairs' float distances: cnt * b * c + sum of the fixed-point offsets
            const long long resid = static_cast<long long>(S.ds[b]) - static_cast<long long>(cnt) * kResBias;
            d = 2.0 * (static_cast<double>(cnt) * b * static_cast<double>(c) +
                       static_cast<double>(resid) / static_cast<double>(scale));
        }
        if (b == 0) {
            v += S.diag_value;
            n += S.diag_count;
        }
        S.out[b] = v;
        S.out[static_cast<size_t>(nb) + b] = n;
        S.out[2 * static_cast<size_t>(nb) + b] = d;
    }
}

}  // namespace

struct Calculator {
    Ctx* ctx = nullptr;
    double bin_width = 0.25;
    int bin_count = 8000;
    struct Set {
        const float* host;  // the caller's array (must stay valid until run)
        int n;
        size_t off;         // first record in `staged`
    };
    std::vector<Set> sets;
    std::vector<float4> staged;
    struct Job {
        int a, b;  // sets; b < 0: self
        int scaling, slot;
    };
    std::vector<Job> jobs;
    std::map<int, int> ids[2];  // self / cross merge id -> slot
    struct SlotInfo {
        int cross, merge_id;
        int index;  // position among the results of its kind (the reference's res_idx)
    };
    std::vector<SlotInfo> slot_info;
    DevBuf points, acc, table, out;
    std::vector<double> results;  // [slots][3][bin_count] of the last run
    std::vector<SlotInfo> result_info;

    int set_of(const float* p, int n) {
        for (size_t k = 0; k < sets.size(); ++k)
            if (sets[k].host == p && sets[k].n == n) return (int)k;
        Set s{p, n, staged.size()};
        staged.resize(staged.size() + n);
        if (n) std::memcpy(staged.data() + s.off, p, (size_t)n * 16);
        sets.push_back(s);
        return (int)sets.size() - 1;
    }

    // SimpleCalculator::enqueue_calculate_self / _cross (SimpleCalculator.h:94-109, 164-181): the
    // result index of the merge id (a new result for a new id; merge id -1: a result of its own,
    // whose id is its index)
    int enqueue(const float* a, int na, const float* b, int nb, int scaling, int merge_id) {
        if (na < 0 || nb < 0 || (na && !a) || (nb && !b)) throw Error{AUSAXS_ERR_ARGUMENT, "invalid point array"};
        if (scaling < 1) throw Error{AUSAXS_ERR_ARGUMENT, "scaling must be positive"};
        const int cross = b != nullptr ? 1 : 0;
        auto& m = ids[cross];
        int slot;
        if (merge_id == -1 || !m.count(merge_id)) {
            const int index = (int)m.size();
            if (merge_id == -1) merge_id = index;
            slot = (int)slot_info.size();
            slot_info.push_back({cross, merge_id, index});
            m[merge_id] = slot;
        } else {
            slot = m[merge_id];
        }
        const int index = slot_info[slot].index;
        jobs.push_back({set_of(a, na), cross ? set_of(b, nb) : -1, scaling, slot});
        return index;
    }

    void run() {
        Ctx& C = *ctx;
        cudaStream_t s = C.stream;
        const int n_slots = (int)slot_info.size();
        results.assign((size_t)n_slots * 3 * bin_count, 0.0);
        result_info = slot_info;
        if (n_slots == 0) return clear();
        // the largest pair distance: min(box diagonal, 2 x radius about the box centre) over all points
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (const float4& p : staged) {
            const double v[3] = {p.x, p.y, p.z};
            for (int d = 0; d < 3; ++d) {
                if (!std::isfinite(v[d])) throw Error{AUSAXS_ERR_ARGUMENT, "non-finite coordinate"};
                lo[d] = std::min(lo[d], v[d]);
                hi[d] = std::max(hi[d], v[d]);
            }
        }
        double dmax = 0;
        if (!staged.empty()) {
            double d2 = 0, r2 = 0, c[3];
            for (int d = 0; d < 3; ++d) {
                d2 += (hi[d] - lo[d]) * (hi[d] - lo[d]);
                c[d] = 0.5 * (lo[d] + hi[d]);
            }
            for (const float4& p : staged) {
                const double e[3] = {p.x - c[0], p.y - c[1], p.z - c[2]};
                r2 = std::max(r2, e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            }
            dmax = std::min(std::sqrt(d2), 2 * std::sqrt(r2)) * (1 + 1e-6) + 1e-3;
        }
        const float inv_w = (float)(1.0 / bin_width);
        int nb = (int)std::ceil(dmax * inv_w) + 2;
        nb = std::max(nb, 11);
        nb = std::min(nb, bin_count);
        if (pairhist_launch_smem(1, nb, true, 512) > kPairSmemCap)
            throw Error{AUSAXS_ERR_CAPACITY, "too many distance bins for the on-chip histogram"};

        // device layout: points, per slot [cnt | ds | ws] (nb each), outputs, slot table, counters
        const size_t pts_bytes = align_up(std::max<size_t>(1, staged.size()) * 16, 256);
        points.ensure(pts_bytes);
        AUSAXS_CUDA(cudaMemcpyAsync(points.p, staged.data(), staged.size() * 16, cudaMemcpyHostToDevice, s));
        const size_t row = align_up((size_t)nb * 8, 256);
        const size_t acc_bytes = (size_t)n_slots * 3 * row + 1024;
        acc.ensure(acc_bytes);
        AUSAXS_CUDA(cudaMemsetAsync(acc.p, 0, acc_bytes, s));
        char* ab = acc.as<char>();
        unsigned long long* counter = reinterpret_cast<unsigned long long*>(ab + (size_t)n_slots * 3 * row);
        unsigned long long* overflow = counter + 4;
        float* wscale = reinterpret_cast<float*>(counter + 8);
        out.ensure((size_t)n_slots * 3 * nb * 8);
        const float4* P = points.as<float4>();
        weight_scale_launch(P, (int)staged.size(), P, 0, wscale, s);
        C.check_launch("calculator weight scale");

        Plan plan;  // job-building view
        plan.T = 1;
        plan.nb = nb;
        plan.inv_w = inv_w;
        plan.c = (float)(1.0 / (double)inv_w);
        plan.scale = (float)(32768.0 / (double)plan.c * (1.0 - 1.0 / 256));
        plan.max_group_rows = 1;
        std::vector<CalcSlot> table_h(n_slots);
        for (int k = 0; k < n_slots; ++k) {
            table_h[k].cnt = reinterpret_cast<unsigned long long*>(ab + (size_t)(3 * k) * row);
            table_h[k].ds = reinterpret_cast<unsigned long long*>(ab + (size_t)(3 * k + 1) * row);
            table_h[k].ws = reinterpret_cast<long long*>(ab + (size_t)(3 * k + 2) * row);
            table_h[k].diag_value = table_h[k].diag_count = 0;
            table_h[k].out = out.as<double>() + (size_t)k * 3 * nb;
        }
        long long pairs = 0;
        int biggest = 0;
        for (const Job& j : jobs) {
            const Set& A = sets[j.a];
            if (j.b < 0) {
                // the diagonal: scaling * sum(float(w*w)) (SimpleCalculator.h:143-161)
                double tw = 0;
                for (int i = 0; i < A.n; ++i) {
                    const float w = staged[A.off + i].w;
                    tw += (double)(float)(w * w);
                }
                tw *= j.scaling;
                table_h[j.slot].diag_value += tw;
                table_h[j.slot].diag_count += (double)(uint32_t)tw;
                if (A.n < 2) continue;
                JobSpec sp{};
                sp.A = sp.B = P + A.off;
                sp.na = sp.nbp = A.n;
                sp.self = 1;
                sp.rmode = kRowSingle;
                sp.rows = 1;
                sp.counts = table_h[j.slot].cnt;
                sp.dsum = table_h[j.slot].ds;
                sp.wsum = table_h[j.slot].ws;
                sp.mult = j.scaling;
                plan.specs.push_back(sp);
                pairs += (long long)A.n * (A.n - 1) / 2;
                biggest = std::max(biggest, A.n);
            } else {
                // enqueue_calculate_cross(data_1 = a, data_2 = b): b outer, a inner from 0
                const Set& B = sets[j.b];
                if (A.n == 0 || B.n == 0) continue;
                JobSpec sp{};
                sp.A = P + B.off;
                sp.na = B.n;
                sp.B = P + A.off;
                sp.nbp = A.n;
                sp.self = 0;
                sp.rmode = kRowSingle;
                sp.rows = 1;
                sp.counts = table_h[j.slot].cnt;
                sp.dsum = table_h[j.slot].ds;
                sp.wsum = table_h[j.slot].ws;
                sp.mult = j.scaling;
                plan.specs.push_back(sp);
                pairs += (long long)A.n * B.n;
                biggest = std::max({biggest, A.n, B.n});
            }
        }
        const size_t table_bytes = align_up(sizeof(CalcSlot) * n_slots, 256);
        std::vector<PairJob> pj[3];
        long long tiles[3] = {0, 0, 0};
        int rows[3] = {1, 1, 1};
        const int tile = biggest >= 16384 ? 512 : 256;
        append_pair_jobs(plan, tile, false, pj, tiles, rows);
        table.ensure(table_bytes + align_up(sizeof(PairJob) * std::max<size_t>(1, pj[0].size()), 256));
        AUSAXS_CUDA(cudaMemcpyAsync(table.p, table_h.data(), sizeof(CalcSlot) * n_slots, cudaMemcpyHostToDevice, s));
        PairJob* jobs_dev = reinterpret_cast<PairJob*>(table.as<char>() + table_bytes);
        if (!pj[0].empty()) {
            AUSAXS_CUDA(cudaMemcpyAsync(jobs_dev, pj[0].data(), sizeof(PairJob) * pj[0].size(), cudaMemcpyHostToDevice, s));
            PairLaunch L{};
            L.jobs = jobs_dev;
            L.n_jobs = (int)pj[0].size();
            L.total_tiles = tiles[0];
            L.smem_rows = 1;
            L.smem_bins = nb;
            L.tile_counter = counter;
            L.overflow = overflow;
            L.weighted = 1;
            L.wscale = wscale;
            L.dreg = 0;
            L.inv_w = plan.inv_w;
            pair_sqrt_prepare(plan.inv_w, nb);
            const size_t smem = pairhist_launch_smem(1, nb, true, tile);
            const int per_sm = pairhist_ctas_per_sm(smem, tile, false, true);
            const int grid = (int)std::min<long long>((long long)C.sm_count * per_sm, std::max<long long>(1, tiles[0]));
            L.chunk = (int)std::max<long long>(1, std::min<long long>(8, tiles[0] / ((long long)grid * 8)));
            cudaEvent_t ev;
            C.time_begin(0, &ev);
            pairhist_launch(L, tile, grid, smem, s);
            C.check_launch("calculator pairs");
            C.time_end(0, ev);
        }
        const int threads = 256;
        calc_finalize_kernel<<<dim3((unsigned)((nb + threads - 1) / threads), (unsigned)n_slots), threads, 0, s>>>(
            reinterpret_cast<const CalcSlot*>(table.p), nb, wscale, plan.c, plan.scale);
        C.check_launch("calculator finalize");
        unsigned long long of = 0;
        AUSAXS_CUDA(cudaMemcpyAsync(&of, overflow, 8, cudaMemcpyDeviceToHost, s));
        std::vector<double> packed((size_t)n_slots * 3 * nb);
        AUSAXS_CUDA(cudaMemcpyAsync(packed.data(), out.p, packed.size() * 8, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaStreamSynchronize(s));
        for (size_t r = 0; r < (size_t)n_slots * 3; ++r)  // [slot][3][nb] -> [slot][3][bin_count]
            std::memcpy(results.data() + r * bin_count, packed.data() + r * nb, (size_t)nb * 8);
        pairs_last = pairs;
        clear();
        if (of)
            throw Error{AUSAXS_ERR_BIN_OVERFLOW, "pair distances beyond bin_count * bin_width; increase settings::axes::bin_count"};
    }

    // SimpleCalculator::run clears its jobs and merge ids (SimpleCalculator.h:278-282)
    void clear() {
        sets.clear();
        staged.clear();
        jobs.clear();
        ids[0].clear();
        ids[1].clear();
        slot_info.clear();
    }

    long long pairs_last = 0;
};

}  // namespace ausaxs_b200

using namespace ausaxs_b200;

struct ausaxs_gpu_calculator {
    Calculator impl;
};

extern "C" {

int ausaxs_gpu_calculator_create(ausaxs_gpu_ctx* ctx, double bin_width, int32_t bin_count, ausaxs_gpu_calculator** out) {
    return guarded([&] {
        if (!ctx || !out || !(bin_width > 0) || bin_count <= 0) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        *out = nullptr;
        auto* c = new ausaxs_gpu_calculator();
        c->impl.ctx = &ctx->impl;
        c->impl.bin_width = bin_width;
        c->impl.bin_count = bin_count;
        *out = c;
    });
}

int ausaxs_gpu_calculator_destroy(ausaxs_gpu_calculator* c) {
    return guarded([&] {
        if (!c) return;
        cudaStreamSynchronize(c->impl.ctx->stream);
        delete c;
    });
}

int ausaxs_gpu_calculator_enqueue_self(ausaxs_gpu_calculator* c, const float* points, int32_t n, int32_t scaling,
                                       int32_t merge_id, int32_t* result_index) {
    return guarded([&] {
        if (!c) throw Error{AUSAXS_ERR_ARGUMENT, "null calculator"};
        const int r = c->impl.enqueue(points, n, nullptr, 0, scaling, merge_id);
        if (result_index) *result_index = r;
    });
}

int ausaxs_gpu_calculator_enqueue_cross(ausaxs_gpu_calculator* c, const float* points_1, int32_t n_1,
                                        const float* points_2, int32_t n_2, int32_t scaling, int32_t merge_id,
                                        int32_t* result_index) {
    return guarded([&] {
        if (!c || (n_2 > 0 && !points_2)) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        // a cross job with an empty second set still creates its (empty) result
        static const float none[4] = {0, 0, 0, 0};
        const int r = c->impl.enqueue(points_1, n_1, points_2 ? points_2 : none, n_2, scaling, merge_id);
        if (result_index) *result_index = r;
    });
}

int ausaxs_gpu_calculator_run(ausaxs_gpu_calculator* c, int32_t* n_self, int32_t* n_cross) {
    return guarded([&] {
        if (!c) throw Error{AUSAXS_ERR_ARGUMENT, "null calculator"};
        AUSAXS_CUDA(cudaSetDevice(c->impl.ctx->device));
        c->impl.run();
        int ns = 0, nc = 0;
        for (auto& r : c->impl.result_info) (r.cross ? nc : ns) += 1;
        if (n_self) *n_self = ns;
        if (n_cross) *n_cross = nc;
    });
}

int ausaxs_gpu_calculator_result_ids(ausaxs_gpu_calculator* c, int32_t cross, int32_t* ids, int32_t capacity, int32_t* n) {
    return guarded([&] {
        if (!c || !n || (capacity > 0 && !ids)) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        std::vector<int> v;
        for (auto& r : c->impl.result_info)
            if (r.cross == (cross != 0)) v.push_back(r.merge_id);
        std::sort(v.begin(), v.end());
        *n = (int32_t)v.size();
        for (int k = 0; k < (int)v.size() && k < capacity; ++k) ids[k] = v[k];
    });
}

int ausaxs_gpu_calculator_result(ausaxs_gpu_calculator* c, int32_t cross, int32_t merge_id, double* value, double* count,
                                 double* distance_sum) {
    return guarded([&] {
        if (!c) throw Error{AUSAXS_ERR_ARGUMENT, "null calculator"};
        const auto& I = c->impl.result_info;
        const size_t nb = c->impl.bin_count;
        for (size_t k = 0; k < I.size(); ++k) {
            if (I[k].cross != (cross != 0) || I[k].merge_id != merge_id) continue;
            const double* r = c->impl.results.data() + k * 3 * nb;
            if (value) std::memcpy(value, r, nb * 8);
            if (count) std::memcpy(count, r + nb, nb * 8);
            if (distance_sum) std::memcpy(distance_sum, r + 2 * nb, nb * 8);
            return;
        }
        throw Error{AUSAXS_ERR_NOT_FOUND, "no result with this merge id in the last run"};
    });
}

}  // extern "C"
