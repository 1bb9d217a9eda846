// hist::distance_calculator::SimpleCalculator over the device calculator (ausaxs_gpu_calculator_*).
//
// Reference-side integration code, compiled against the reference's headers: a translation unit of
// the reference (SymmetryManagerMT.cpp, PartialSymmetryManagerMT.cpp) compiled with this directory
// first on its include path gets this class in place of the thread-pool calculator of
// include/core/hist/distance_calculator/SimpleCalculator.h:37-92, with the same members, arguments
// and results, so the reference's symmetry managers issue their pair work to the GPU unchanged.  The
// class lives in an inline namespace: its symbols differ from the CPU calculator's, which other
// reference translation units of the same library still use.
#pragma once

#include <hist/detail/CompactCoordinates.h>
#include <hist/distribution/GenericDistribution1D.h>
#include <settings/HistogramSettings.h>

#include <ausaxs_b200.h>

#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace ausaxs::hist::distance_calculator {
inline namespace gpu {
    // the process-wide device context of the adapter (oracle/adapter/gpu_adapter.cpp)
    ausaxs_gpu_ctx* adapter_context();

    inline void adapter_check(int rc) {
        if (rc != AUSAXS_OK) throw std::runtime_error(std::string("ausaxs_b200: ") + ausaxs_gpu_last_error());
    }

    template<bool weighted_bins, bool variable_bin_width>
    class SimpleCalculator {
        using GenericDistribution1D_t = typename hist::GenericDistribution1D<weighted_bins>::type;
        public:
            struct run_result {
                std::unordered_map<int, GenericDistribution1D_t> self;
                std::unordered_map<int, GenericDistribution1D_t> cross;
            };

            SimpleCalculator() {
                adapter_check(ausaxs_gpu_calculator_create(adapter_context(), settings::axes::bin_width,
                                                           (int32_t)settings::axes::bin_count, &c));
            }
            ~SimpleCalculator() { if (c) ausaxs_gpu_calculator_destroy(c); }
            SimpleCalculator(const SimpleCalculator&) = delete;
            SimpleCalculator& operator=(const SimpleCalculator&) = delete;

            int enqueue_calculate_self(const hist::detail::CompactCoordinates<variable_bin_width>& a, int scaling = 1, int merge_id = -1) {
                int32_t r = 0;
                adapter_check(ausaxs_gpu_calculator_enqueue_self(c, raw(a), (int32_t)a.size(), scaling, merge_id, &r));
                n_self = std::max(n_self, r + 1);
                return r;
            }

            int enqueue_calculate_cross(const hist::detail::CompactCoordinates<variable_bin_width>& a1,
                                        const hist::detail::CompactCoordinates<variable_bin_width>& a2, int scaling = 1, int merge_id = -1) {
                int32_t r = 0;
                adapter_check(ausaxs_gpu_calculator_enqueue_cross(c, raw(a1), (int32_t)a1.size(), raw(a2), (int32_t)a2.size(),
                                                                  scaling, merge_id, &r));
                n_cross = std::max(n_cross, r + 1);
                return r;
            }

            int size_self_result() const { return n_self; }
            int size_cross_result() const { return n_cross; }

            run_result run() {
                adapter_check(ausaxs_gpu_calculator_run(c, nullptr, nullptr));
                run_result out;
                collect(0, out.self);
                collect(1, out.cross);
                n_self = n_cross = 0;
                return out;
            }

        private:
            ausaxs_gpu_calculator* c = nullptr;
            int n_self = 0, n_cross = 0;

            static const float* raw(const hist::detail::CompactCoordinates<variable_bin_width>& a) {
                static_assert(sizeof(a.get_data()[0]) == 16, "compact coordinates are 16-byte {x, y, z, w} records");
                return reinterpret_cast<const float*>(a.get_data().data());
            }

            // every result of one kind as the reference's distributions (value, count, distance sum per bin)
            void collect(int cross, std::unordered_map<int, GenericDistribution1D_t>& into) {
                int32_t n = 0;
                adapter_check(ausaxs_gpu_calculator_result_ids(c, cross, nullptr, 0, &n));
                std::vector<int32_t> ids(n);
                if (n) adapter_check(ausaxs_gpu_calculator_result_ids(c, cross, ids.data(), n, &n));
                const int nb = (int)settings::axes::bin_count;
                std::vector<double> value(nb), count(nb), dsum(nb);
                for (int32_t id : ids) {
                    adapter_check(ausaxs_gpu_calculator_result(c, cross, id, value.data(), count.data(), dsum.data()));
                    GenericDistribution1D_t d(nb);
                    for (int b = 0; b < nb; ++b) {
                        if constexpr (weighted_bins) {
                            d.index(b) = hist::detail::WeightedEntry(value[b], (unsigned int)count[b], dsum[b]);
                        } else {
                            d.index(b) = value[b];
                        }
                    }
                    into.emplace(id, std::move(d));
                }
            }
    };
}
}
