// Reference-side integration code: a histogram manager of the reference (hist::IHistogramManager,
// include/core/hist/histogram_manager/IHistogramManager.h:16-29) whose calculate_all() runs on the
// device through the C ABI of include/ausaxs_b200.h and returns the reference's own
// CompositeDistanceHistogramFFAvg, built as HistogramManagerMTFFAvg::calculate_all() builds it
// (source/core/hist/histogram_manager/HistogramManagerMTFFAvg.cpp:304-371): raw counts by
// form-factor pair (excluded-volume rows scaled by Z_exv), the total with its weighted distance axis,
// cut at the last non-zero bin.  Everything downstream (debye_transform, the fitters) is the
// reference's code.  Compiled against the reference's headers (oracle/Makefile, target `adapter`).
#pragma once

#include <constants/Constants.h>
#include <settings/FormFactorSettings.h>
#include <data/Molecule.h>
#include <hist/detail/CompactCoordinatesFF.h>
#include <hist/distribution/Distribution1D.h>
#include <hist/distribution/Distribution2D.h>
#include <hist/distribution/Distribution3D.h>
#include <hist/distribution/WeightedDistribution1D.h>
#include <hist/histogram_manager/HistogramManager.h>
#include <hist/intensity_calculator/CompositeDistanceHistogramFFAvg.h>
#include <settings/HistogramSettings.h>

#include <ausaxs_b200.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace ausaxs::hist::distance_calculator {
inline namespace gpu {
    ausaxs_gpu_ctx* adapter_context();
}
}

namespace ausaxs::hist {
    template<bool variable_bin_width>
    class GpuHistogramManagerMTFFAvg : public HistogramManager<true, variable_bin_width> {
        public:
            using HistogramManager<true, variable_bin_width>::HistogramManager;

            std::unique_ptr<DistanceHistogram> calculate() override { return calculate_all(); }

            std::unique_ptr<ICompositeDistanceHistogram> calculate_all() override {
                const data::Molecule& m = *this->protein;
                detail::CompactCoordinatesFF<variable_bin_width> a(m.get_bodies()), w(m.get_waters());
                const double z_exv = m.size_atom() == 0 ? 0 : m.get_volume_grid() * constants::charge::density::water / m.size_atom();
                ausaxs_hist_config cfg{AUSAXS_MANAGER_FFAVG, 1, settings::axes::bin_width, (int32_t)settings::axes::bin_count, z_exv};
                const int nb = (int)settings::axes::bin_count, nff = (int)settings::form_factor::max_ff_types;
                std::vector<double> aa((size_t)nff * nff * nb), aw((size_t)nff * nb), ww(nb), tot(nb), d(nb);
                ausaxs_hist_result r{};
                r.aa = aa.data();
                r.aw = aw.data();
                r.ww = ww.data();
                r.tot = tot.data();
                r.d_axis = d.data();
                check(ausaxs_gpu_histogram(distance_calculator::adapter_context(), &cfg,
                                           reinterpret_cast<const float*>(a.get_data().data()), (int32_t)a.size(),
                                           reinterpret_cast<const float*>(w.get_data().data()), (int32_t)w.size(),
                                           nullptr, 0, &r));
                const int mb = r.max_bin;
                Distribution3D p_aa(nff, nff, mb);
                Distribution2D p_aw(nff, mb);
                Distribution1D p_ww(mb);
                WeightedDistribution1D p_tot(mb);
                for (int i = 0; i < nff; ++i) {
                    for (int j = 0; j < nff; ++j)
                        for (int b = 0; b < mb; ++b) p_aa.index(i, j, b) = aa[((size_t)i * nff + j) * mb + b];
                    for (int b = 0; b < mb; ++b) p_aw.index(i, b) = aw[(size_t)i * mb + b];
                }
                for (int b = 0; b < mb; ++b) {
                    p_ww.index(b) = ww[b];
                    // the weighted axis as the entry's distance sum over a unit count; empty bins keep
                    // the reference's b * width
                    p_tot.index(b) = tot[b] != 0 ? detail::WeightedEntry(tot[b], 1, d[b]) : detail::WeightedEntry(0, 0, 0);
                }
                return std::make_unique<CompositeDistanceHistogramFFAvg>(std::move(p_aa), std::move(p_aw), std::move(p_ww),
                                                                         std::move(p_tot));
            }

        private:
            static void check(int rc) {
                if (rc != AUSAXS_OK) throw std::runtime_error(std::string("ausaxs_b200: ") + ausaxs_gpu_last_error());
            }
    };
}
