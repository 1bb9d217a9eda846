// C entry points over the reference implementation, compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/libausaxs_ref.so.
//
// Test infrastructure only: the parity tests call it (through ctypes) to pin
// the C restatement in oracle/oracle.c and the CUDA path, and bench.py's
// reference arm times it as the CPU baseline.  Nothing in the product links it.
//
// Every function drives the reference's public C++ API exactly as its own
// tests do (tests/feature/hist/hist_test_helper.h:19-27 for the volume-scaled
// molecule; histogram_manager.cpp:74-190 for the managers).  Arrays are
// row-major FP64, sizes are explicit, errors come back as a non-zero int with
// the message in ref_last_error().
#include <map>

#include <data/Body.h>
#include <data/Molecule.h>
#include <data/atoms/AtomFF.h>
#include <data/atoms/Water.h>
#include <dataset/SimpleDataset.h>
#include <fitter/detail/LinearLeastSquares.h>
#include <fitter/FitResult.h>
#include <fitter/SmartFitter.h>
#include <settings/FitSettings.h>
#include <grid/detail/GridExcludedVolume.h>
#include <hist/detail/SimpleExvModel.h>
#include <hist/distance_calculator/SimpleCalculator.h>
#include <hist/distribution/Distribution1D.h>
#include <hist/distribution/WeightedDistribution1D.h>
#include <hist/distribution/Distribution2D.h>
#include <hist/distribution/Distribution3D.h>
#include <hist/histogram_manager/HistogramManager.h>
#include <hist/histogram_manager/HistogramManagerMT.h>
#include <hist/histogram_manager/HistogramManagerMTFFAvg.h>
#include <hist/histogram_manager/HistogramManagerMTFFExplicit.h>
#include <hist/histogram_manager/HistogramManagerMTFFGrid.h>
#include <hist/histogram_manager/PartialHistogramManagerMT.h>
#include <hist/histogram_manager/SymmetryManagerMT.h>
#include <data/symmetry/PredefinedSymmetries.h>
#include <data/symmetry/CompositeSymmetry.h>
#include <hist/intensity_calculator/CompositeDistanceHistogramFFGrid.h>
#include <hist/intensity_calculator/DistanceHistogram.h>
#include <hist/intensity_calculator/ExactDebyeCalculator.h>
#include <hist/intensity_calculator/ICompositeDistanceHistogram.h>
#include <hist/intensity_calculator/ICompositeDistanceHistogramExv.h>
#include <math/Matrix.h>
#include <settings/ExvSettings.h>
#include <settings/Flags.h>
#include <settings/GeneralSettings.h>
#include <settings/HistogramSettings.h>
#include <settings/MoleculeSettings.h>
#include <settings/GridSettings.h>
#include <grid/Grid.h>
#include <grid/exv/RawGridExv.h>
#include <grid/detail/GridMember.h>
#include <hydrate/generation/RadialHydration.h>
#include <hydrate/generation/HydrationStrategy.h>
#include <io/File.h>

#ifdef AUSAXS_ADAPTER
#include "adapter/gpu_adapter.h"
#endif

#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace ausaxs;

namespace {
thread_local std::string g_err;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
    } catch (...) {
        g_err = "unknown exception";
    }
    return 1;
}

// A molecule whose excluded volume is given instead of derived from the
// reference's voxel grid, as the reference's own DebugMolecule does.
class FixedVolumeMolecule : public data::Molecule {
  public:
    using Molecule::Molecule;
    double get_volume_grid() const override { return volume >= 0 ? volume : data::Molecule::get_volume_grid(); }
    double volume = -1;
};

// The grid manager with its excluded-volume dummies supplied by the caller
// (HistogramManagerMTFFGrid::get_exv is the one virtual hook for them).
template <bool vbw>
class GivenExvGridManager : public hist::HistogramManagerMTFFGrid<vbw> {
  public:
    GivenExvGridManager(observer_ptr<const data::Molecule> m, std::vector<Vector3<double>> x)
        : hist::HistogramManagerMTFFGrid<vbw>(m), exv(std::move(x)) {}

  private:
    grid::exv::GridExcludedVolume get_exv() const override {
        grid::exv::GridExcludedVolume g;
        g.interior = exv;
        return g;
    }
    std::vector<Vector3<double>> exv;
};

struct Result {
    std::unique_ptr<hist::ICompositeDistanceHistogram> h;
    int kind = 0;
};

bool custom_width() { return settings::flags::custom_bin_width; }

// The calculator on the width instantiation the managers would pick (custom bin width: variable).
template <bool vbw>
void run_calculator(const double* pts, const int* set_off, int n_sets, int n_jobs, const int* ja, const int* jb,
                    const int* scaling, const int* merge, int* n_results, int* keys, double* out) {
    std::vector<hist::detail::CompactCoordinates<vbw>> sets;
    sets.reserve(n_sets);
    for (int s = 0; s < n_sets; ++s) {
        std::vector<data::Water> w;
        for (int i = set_off[s]; i < set_off[s + 1]; ++i) w.emplace_back(Vector3<double>(pts[4 * i], pts[4 * i + 1], pts[4 * i + 2]));
        sets.emplace_back(w);
        auto& d = sets.back().get_data();
        for (int i = set_off[s]; i < set_off[s + 1]; ++i) {
            auto& e = d[i - set_off[s]];
            e.value.pos = Vector3<float>(pts[4 * i], pts[4 * i + 1], pts[4 * i + 2]);
            e.value.w = static_cast<float>(pts[4 * i + 3]);
        }
    }
    hist::distance_calculator::SimpleCalculator<true, vbw> calc;
    for (int k = 0; k < n_jobs; ++k) {
        if (jb[k] < 0) calc.enqueue_calculate_self(sets[ja[k]], scaling[k], merge[k]);
        else calc.enqueue_calculate_cross(sets[ja[k]], sets[jb[k]], scaling[k], merge[k]);
    }
    auto res = calc.run();
    const size_t nb = settings::axes::bin_count;
    int r = 0;
    auto put = [&](int cross, std::map<int, const hist::WeightedDistribution1D*>& m) {
        for (auto& [id, dist] : m) {
            keys[2 * r] = cross;
            keys[2 * r + 1] = id;
            for (size_t i = 0; i < nb && i < dist->size(); ++i) {
                const auto& e = dist->index(i);
                out[(3 * r + 0) * nb + i] = e.value;
                out[(3 * r + 1) * nb + i] = e.count;
                out[(3 * r + 2) * nb + i] = e.bin_center;
            }
            ++r;
        }
    };
    std::map<int, const hist::WeightedDistribution1D*> self, cross;
    for (auto& [id, d] : res.self) self[id] = &d;
    for (auto& [id, d] : res.cross) cross[id] = &d;
    put(0, self);
    put(1, cross);
    *n_results = r;
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// Must be called before any other entry point: sizes the reference's global
// thread pool (settings::general::threads, read once at first use).
int ref_init(int threads) {
    return guarded([&] {
        settings::general::threads = threads > 0 ? threads : 1;
        settings::flags::init_histogram_manager = false;
        settings::general::verbose = false;
        settings::general::warnings = false;
    });
}

int ref_set_axes(double bin_width, int bin_count, double qmin, double qmax) {
    return guarded([&] {
        settings::axes::bin_count = static_cast<unsigned int>(bin_count);
        settings::axes::bin_width = bin_width;
        settings::axes::qmin = qmin;
        settings::axes::qmax = qmax;
    });
}

int ref_set_simple_exv(int enable) {
    return guarded([&] {
        if (enable) hist::detail::SimpleExvModel::enable();
        else hist::detail::SimpleExvModel::disable();
    });
}

// atoms: n_a rows of {x, y, z, weight, ff_type}; waters: n_w rows of {x, y, z, weight}.
// body_sizes splits the atoms into consecutive bodies (n_bodies >= 1); all
// waters go to the first body.  volume < 0 keeps the reference's own grid volume.
void* ref_molecule_new(const double* atoms, int n_a, const double* waters, int n_w,
                       const int* body_sizes, int n_bodies, double volume) {
    FixedVolumeMolecule* out = nullptr;
    int rc = guarded([&] {
        std::vector<data::Body> bodies;
        int off = 0;
        int nb = n_bodies > 0 ? n_bodies : 1;
        for (int b = 0; b < nb; ++b) {
            int sz = n_bodies > 0 ? body_sizes[b] : n_a;
            std::vector<data::AtomFF> a;
            a.reserve(sz);
            for (int i = off; i < off + sz; ++i) {
                const double* r = atoms + 5 * static_cast<size_t>(i);
                a.emplace_back(Vector3<double>(r[0], r[1], r[2]), static_cast<form_factor::form_factor_t>(static_cast<int>(r[4])), r[3]);
            }
            off += sz;
            std::vector<data::Water> w;
            if (b == 0) {
                w.reserve(n_w);
                for (int i = 0; i < n_w; ++i) {
                    const double* r = waters + 4 * static_cast<size_t>(i);
                    data::Water x(Vector3<double>(r[0], r[1], r[2]));
                    x.weight() = r[3];
                    w.push_back(x);
                }
            }
            bodies.emplace_back(std::move(a), std::move(w));
        }
        out = new FixedVolumeMolecule(std::move(bodies));
        out->volume = volume;
    });
    return rc == 0 ? out : nullptr;
}

void ref_molecule_free(void* m) { delete static_cast<FixedVolumeMolecule*>(m); }

// RawGridExv::create on the molecule's expanded grid, as HistogramManagerMTFFGrid::calculate_all()
// uses it (get_volume_grid() expands first): atoms n x {x, y, z, ff}, waters n x {x, y, z}; writes
// up to cap dummies n x {x, y, z}.  settings::grid::scaling is reset to its default first: the
// reference's Grid constructor sets it to 1 for small structures and leaves it so for later grids.
int ref_grid_exv(const double* atoms, int n_a, const double* waters, int n_w, double* out, int cap, int* n_out,
                 double* volume) {
    return guarded([&] {
        settings::grid::scaling = 0.25;
        std::vector<data::AtomFF> a;
        for (int i = 0; i < n_a; ++i) {
            const double* r = atoms + 4 * static_cast<size_t>(i);
            a.emplace_back(Vector3<double>(r[0], r[1], r[2]), static_cast<form_factor::form_factor_t>(static_cast<int>(r[3])));
        }
        std::vector<data::Water> w;
        for (int i = 0; i < n_w; ++i) {
            const double* r = waters + 3 * static_cast<size_t>(i);
            w.emplace_back(Vector3<double>(r[0], r[1], r[2]));
        }
        std::vector<data::Body> bodies;
        bodies.emplace_back(std::move(a), std::move(w));
        data::Molecule m(std::move(bodies));
        *volume = m.get_volume_grid();
        auto exv = grid::exv::RawGridExv::create(m.get_grid()).interior;
        *n_out = static_cast<int>(exv.size());
        if (out && cap >= *n_out)
            for (size_t i = 0; i < exv.size(); ++i) {
                out[3 * i] = exv[i].x();
                out[3 * i + 1] = exv[i].y();
                out[3 * i + 2] = exv[i].z();
            }
    });
}

// A structure file read by the reference's own reader (data::Molecule(io::File), which assigns the
// united-atom form-factor types), returned as arrays: atoms n x {x, y, z, weight, ff}, waters
// n x {x, y, z, weight}.  Call with capacities 0 to get the counts.  implicit_hydrogens and center
// take the reference's defaults unless set to 0 / 1 explicitly (-1: default).
int ref_read_structure(const char* path, int implicit_h, int center, double* atoms, int cap_a, int* n_a, double* waters,
                       int cap_w, int* n_w) {
    return guarded([&] {
        if (implicit_h >= 0) settings::molecule::implicit_hydrogens = implicit_h != 0;
        if (center >= 0) settings::molecule::center = center != 0;
        data::Molecule m{io::File(std::string(path))};
        auto a = m.get_atoms();
        auto w = m.get_waters();
        *n_a = static_cast<int>(a.size());
        *n_w = static_cast<int>(w.size());
        if (atoms && cap_a >= *n_a) {
            for (size_t i = 0; i < a.size(); ++i) {
                double* r = atoms + 5 * i;
                r[0] = a[i].coordinates().x();
                r[1] = a[i].coordinates().y();
                r[2] = a[i].coordinates().z();
                r[3] = a[i].weight();
                r[4] = static_cast<int>(a[i].form_factor_type());
            }
        }
        if (waters && cap_w >= *n_w) {
            for (size_t i = 0; i < w.size(); ++i) {
                double* r = waters + 4 * i;
                r[0] = w[i].coordinates().x();
                r[1] = w[i].coordinates().y();
                r[2] = w[i].coordinates().z();
                r[3] = w[i].weight();
            }
        }
    });
}

// Rigid move of one body: x <- R x + t, through Body::rotate / Body::translate
// (source/core/data/Body.cpp:135-156), which also signal the partial managers.
// A predefined symmetry (symmetry::create: "c3", "d2", "tetrahedral", "icosahedral", "p2", ...) on a body,
// its leaves' first translation and rotation parameters set as the reference's own tests set them
// (tests/feature/hist/symmetries/symmetry_body_frame.cpp:99-109).
int ref_body_add_symmetry(void* m, int body, const char* name, double translation, double rotation) {
    return guarded([&] {
        auto* mol = static_cast<FixedVolumeMolecule*>(m);
        if (body < 0 || body >= (int)mol->size_body()) throw std::runtime_error("no such body");
        auto sym = symmetry::create(name);
        symmetry::for_each_leaf(*sym, [translation, rotation](symmetry::ISymmetry& leaf) {
            auto t = leaf.span_translation();
            auto r = leaf.span_rotation();
            if (!t.empty()) t[0] = translation;
            if (!r.empty()) r[0] = rotation;
        });
        mol->get_body(body).symmetry().add(std::move(sym));
    });
}

// Whether this build runs the symmetry, Simple and partial managers' pair work on the device.
int ref_adapter_build() {
#ifdef AUSAXS_ADAPTER
    return 1;
#else
    return 0;
#endif
}

int ref_body_move(void* m, int body, const double* R, const double* t) {
    return guarded([&] {
        auto* mol = static_cast<FixedVolumeMolecule*>(m);
        auto& b = mol->get_body(body);
        Matrix<double> M{{R[0], R[1], R[2]}, {R[3], R[4], R[5]}, {R[6], R[7], R[8]}};
        b.rotate(M);
        b.translate(Vector3<double>(t[0], t[1], t[2]));
    });
}

// Hydration: Molecule::generate_new_hydration() with the default strategy (RadialHydration, no
// culling), its noise generator reading successive rows of `noise` (n x 3; zero once exhausted or
// when noise is null).  fresh_grid = 1 drops the molecule's grid and generator first, so the grid
// is rebuilt from the current atoms (Grid(bodies), with settings::grid::scaling back at its default);
// 0 keeps both, as the rigid-body loop does between steps.  Writes the grid's member atoms in the
// order the generator visits them (n_a x {x, y, z, ff}), the waters of every body in body order
// (n_w x 3), the waters per body, and the grid axes {min x, y, z, max x, y, z, bins x, y, z}.
namespace {
std::vector<double> g_noise;
size_t g_noise_at = 0;
}  // namespace

int ref_hydrate(void* m, const double* noise, int n_noise, int fresh_grid, double* atoms_out, int cap_a, int* n_a,
                double* waters_out, int cap_w, int* n_w, int* per_body, double* axes_out) {
    return guarded([&] {
        auto* mol = static_cast<FixedVolumeMolecule*>(m);
        settings::hydrate::hydration_strategy = settings::hydrate::HydrationStrategy::RadialStrategy;
        settings::hydrate::culling_strategy = settings::hydrate::CullingStrategy::NoStrategy;
        g_noise.assign(noise ? noise : nullptr, noise ? noise + 3 * static_cast<size_t>(n_noise) : nullptr);
        g_noise_at = 0;
        hydrate::RadialHydration::set_noise_generator([] {
            if (3 * g_noise_at + 2 >= g_noise.size()) return Vector3<double>(0, 0, 0);
            const double* r = g_noise.data() + 3 * g_noise_at++;
            return Vector3<double>(r[0], r[1], r[2]);
        });
        if (fresh_grid) {
            settings::grid::scaling = 0.25;
            mol->clear_hydration();
            mol->clear_grid();
            mol->set_hydration_generator(nullptr);
        }
        mol->generate_new_hydration();
        auto* grid = mol->get_grid();
        *n_a = static_cast<int>(grid->a_members.size());
        if (atoms_out && cap_a >= *n_a) {
            for (size_t i = 0; i < grid->a_members.size(); ++i) {
                const auto& a = grid->a_members[i].get_atom();
                double* r = atoms_out + 4 * i;
                r[0] = a.coordinates().x();
                r[1] = a.coordinates().y();
                r[2] = a.coordinates().z();
                r[3] = static_cast<int>(a.form_factor_type());
            }
        }
        auto w = mol->get_waters();
        *n_w = static_cast<int>(w.size());
        if (waters_out && cap_w >= *n_w) {
            for (size_t i = 0; i < w.size(); ++i) {
                waters_out[3 * i] = w[i].coordinates().x();
                waters_out[3 * i + 1] = w[i].coordinates().y();
                waters_out[3 * i + 2] = w[i].coordinates().z();
            }
        }
        if (per_body)
            for (size_t b = 0; b < mol->size_body(); ++b) {
                auto h = mol->get_body(b).get_waters();
                per_body[b] = h.has_value() ? static_cast<int>(h.value().get().size()) : 0;
            }
        if (axes_out) {
            const auto& ax = grid->get_axes();
            const Axis* a3[3] = {&ax.x, &ax.y, &ax.z};
            for (int d = 0; d < 3; ++d) {
                axes_out[d] = a3[d]->min;
                axes_out[3 + d] = a3[d]->max;
                axes_out[6 + d] = a3[d]->bins;
            }
        }
    });
}

// A rigid move of one body as the rigid-body transforms make it (SingleTransform.cpp:20-69): the body
// leaves the grid, moves (x <- R x + t) and is added back, which appends its atoms to the grid's
// member list; the grid's axes are kept.
int ref_body_move_in_grid(void* m, int body, const double* R, const double* t) {
    return guarded([&] {
        auto* mol = static_cast<FixedVolumeMolecule*>(m);
        auto& b = mol->get_body(body);
        mol->get_grid()->remove(b);
        Matrix<double> M{{R[0], R[1], R[2]}, {R[3], R[4], R[5]}, {R[6], R[7], R[8]}};
        b.rotate(M);
        b.translate(Vector3<double>(t[0], t[1], t[2]));
        mol->get_grid()->add(b);
    });
}

// The current coordinates of a body's atoms, or with body = -1 of the molecule's waters (which the
// bodies own and move with them, Body.cpp:135-156): n x 3 doubles; out may be null to query n.
int ref_body_coords(void* m, int body, double* out, int* n) {
    return guarded([&] {
        auto* mol = static_cast<FixedVolumeMolecule*>(m);
        auto put = [&](const auto& items) {
            *n = static_cast<int>(items.size());
            if (!out) return;
            for (size_t i = 0; i < items.size(); ++i) {
                const auto& c = items[i].coordinates();
                out[3 * i] = c.x();
                out[3 * i + 1] = c.y();
                out[3 * i + 2] = c.z();
            }
        };
        if (body < 0) put(mol->get_waters());
        else put(mol->get_body(body).get_atoms());
    });
}

// manager: 0 HistogramManager (1 thread), 1 HistogramManagerMT, 2 MTFFAvg,
// 3 MTFFExplicit, 4 MTFFGrid (exv dummies given), 5 PartialHistogramManagerMT.
// The manager is installed in the molecule (Molecule::set_histogram_manager,
// which binds the body signallers the partial manager listens to);
// ref_manager_calculate then runs Molecule::get_histogram().
int ref_manager_set(void* m, int manager, int weighted_bins, const double* exv, int n_x) {
    return guarded([&] {
        hist::IHistogramManager* out = nullptr;
        auto* mol = static_cast<FixedVolumeMolecule*>(m);
        bool vbw = custom_width();
        bool wb = weighted_bins != 0;
        std::vector<Vector3<double>> x;
        for (int i = 0; i < n_x; ++i) x.emplace_back(exv[3 * i], exv[3 * i + 1], exv[3 * i + 2]);
#define PICK(T)                                                                   \
    if (wb) out = vbw ? (hist::IHistogramManager*)new T<true, true>(mol)          \
                      : (hist::IHistogramManager*)new T<true, false>(mol);        \
    else out = vbw ? (hist::IHistogramManager*)new T<false, true>(mol)            \
                   : (hist::IHistogramManager*)new T<false, false>(mol);
        switch (manager) {
            case 0: PICK(hist::HistogramManager); break;
            case 1: PICK(hist::HistogramManagerMT); break;
            case 2: PICK(hist::HistogramManagerMTFFAvg); break;
            case 3: PICK(hist::HistogramManagerMTFFExplicit); break;
            case 4:
                out = vbw ? (hist::IHistogramManager*)new GivenExvGridManager<true>(mol, std::move(x))
                          : (hist::IHistogramManager*)new GivenExvGridManager<false>(mol, std::move(x));
                break;
            case 5: PICK(hist::PartialHistogramManagerMT); break;
            case 6: PICK(hist::SymmetryManagerMT); break;
#ifdef AUSAXS_ADAPTER
            case 7:  // the device FFAvg manager of the adapter (weighted bins)
                out = vbw ? (hist::IHistogramManager*)new hist::GpuHistogramManagerMTFFAvg<true>(mol)
                          : (hist::IHistogramManager*)new hist::GpuHistogramManagerMTFFAvg<false>(mol);
                break;
#endif
            default: throw std::runtime_error("unknown manager");
        }
#undef PICK
        mol->set_histogram_manager(std::unique_ptr<hist::IHistogramManager>(out));
    });
}

void* ref_manager_calculate(void* m, double* seconds) {
    Result* out = nullptr;
    int rc = guarded([&] {
        auto t0 = std::chrono::steady_clock::now();
        auto h = static_cast<FixedVolumeMolecule*>(m)->get_histogram();
        auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        out = new Result{std::move(h), 0};
    });
    return rc == 0 ? out : nullptr;
}

void ref_hist_free(void* r) { delete static_cast<Result*>(r); }

int ref_hist_bins(void* r) { return static_cast<int>(static_cast<Result*>(r)->h->get_d_axis().size()); }

int ref_hist_total(void* r, double* counts, double* d_axis) {
    return guarded([&] {
        auto* h = static_cast<Result*>(r)->h.get();
        const auto& c = h->get_weighted_counts();
        const auto& d = h->get_d_axis();
        std::memcpy(counts, c.data(), c.size() * sizeof(double));
        std::memcpy(d_axis, d.data(), d.size() * sizeof(double));
    });
}

// Simple (weights) composite: aa, aw, ww weighted counts, each bins long.
int ref_hist_simple(void* r, double* aa, double* aw, double* ww) {
    return guarded([&] {
        auto* h = static_cast<Result*>(r)->h.get();
        const auto& a = h->get_aa_counts();
        const auto& b = h->get_aw_counts();
        const auto& c = h->get_ww_counts();
        for (size_t i = 0; i < a.size(); ++i) aa[i] = a.index(i);
        for (size_t i = 0; i < b.size(); ++i) aw[i] = b.index(i);
        for (size_t i = 0; i < c.size(); ++i) ww[i] = c.index(i);
    });
}

// Form-factor composites: raw aa [15][15][bins], aw [15][bins], ww [bins].
int ref_hist_ff(void* r, double* aa, double* aw, double* ww) {
    return guarded([&] {
        auto* h = dynamic_cast<hist::ICompositeDistanceHistogramExv*>(static_cast<Result*>(r)->h.get());
        if (!h) throw std::runtime_error("not a form-factor histogram");
        const auto& a = h->get_raw_aa_counts_by_ff();
        const auto& b = h->get_raw_aw_counts_by_ff();
        const auto& c = h->get_raw_ww_counts_by_ff();
        size_t nb = c.size();
        for (size_t i = 0; i < 15; ++i)
            for (size_t j = 0; j < 15; ++j)
                for (size_t k = 0; k < nb; ++k) aa[(i * 15 + j) * nb + k] = a.index(i, j, k);
        for (size_t i = 0; i < 15; ++i)
            for (size_t k = 0; k < nb; ++k) aw[i * nb + k] = b.index(i, k);
        for (size_t k = 0; k < nb; ++k) ww[k] = c.index(k);
    });
}

// Grid composite: the extra ax and xx weighted distance axes (bins long).
int ref_hist_grid_axes(void* r, double* ax, double* xx) {
    return guarded([&] {
        auto* h = dynamic_cast<hist::CompositeDistanceHistogramFFGrid*>(static_cast<Result*>(r)->h.get());
        if (!h) throw std::runtime_error("not a grid histogram");
        const auto& a = h->get_d_axis_ax();
        const auto& x = h->get_d_axis_xx();
        std::memcpy(ax, a.data(), a.size() * sizeof(double));
        std::memcpy(xx, x.data(), x.size() * sizeof(double));
    });
}

int ref_hist_grid_axis_sizes(void* r, int* n_ax, int* n_xx) {
    return guarded([&] {
        auto* h = dynamic_cast<hist::CompositeDistanceHistogramFFGrid*>(static_cast<Result*>(r)->h.get());
        if (!h) throw std::runtime_error("not a grid histogram");
        *n_ax = static_cast<int>(h->get_d_axis_ax().size());
        *n_xx = static_cast<int>(h->get_d_axis_xx().size());
    });
}

// debye_transform() on the reference's default q axis restricted to
// [qmin, qmax].  For form-factor histograms the six partial profiles
// {aa, ax, aw, xx, wx, ww} are written to profiles (6 x nq) when non-null;
// for the Simple histogram {aa, aw, ww} go to rows 0, 2, 5.
int ref_debye(void* r, double cw, double cx, double crho, double dw_atomic, double dw_exv,
              double* q_out, double* Iq, double* profiles, int* nq, double* seconds) {
    return guarded([&] {
        auto* h = static_cast<Result*>(r)->h.get();
        h->apply_water_scaling_factor(cw);
        auto* x = dynamic_cast<hist::ICompositeDistanceHistogramExv*>(h);
        if (x) {
            x->apply_excluded_volume_scaling_factor(cx);
            x->apply_solvent_density_scaling_factor(crho);
            x->apply_atomic_debye_waller_factor(dw_atomic);
            x->apply_exv_debye_waller_factor(dw_exv);
        }
        auto t0 = std::chrono::steady_clock::now();
        auto I = h->debye_transform();
        auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        const auto& c = I.get_counts();
        auto qv = I.get_axis().as_vector();
        *nq = static_cast<int>(c.size());
        if (Iq) std::memcpy(Iq, c.data(), c.size() * sizeof(double));
        if (q_out) std::memcpy(q_out, qv.data(), qv.size() * sizeof(double));
        if (profiles) {
            size_t n = c.size();
            auto put = [&](int row, const hist::ScatteringProfile& p) {
                const auto& v = p.get_counts();
                std::memcpy(profiles + row * n, v.data(), n * sizeof(double));
            };
            std::memset(profiles, 0, 6 * n * sizeof(double));
            put(0, h->get_profile_aa());
            put(2, h->get_profile_aw());
            put(5, h->get_profile_ww());
            if (x) {
                put(1, x->get_profile_ax());
                put(3, x->get_profile_xx());
                put(4, x->get_profile_wx());
            }
        }
    });
}

// fitter::SmartFitter::fit() (source/core/fitter/SmartFitter.cpp:147-176) with one enabled parameter
// (param 0 water scaling, 1 excluded-volume scaling, 2 solvent density, 3 atomic Debye-Waller, 4 exv
// Debye-Waller) and the default minimiser of a build without dlib (mini::Golden), on the data
// (q, I, sigma).  Consumes the histogram.  out = {value, a, b, chi2, fevals, seconds of fit()}.
int ref_fit(void* r, int param, const double* q, const double* I, const double* sigma, int n, double* out) {
    return guarded([&] {
        using sf = settings::fit;
        sf::fit_hydration = param == 0;
        sf::fit_excluded_volume = param == 1;
        sf::fit_solvent_density = param == 2;
        sf::fit_atomic_debye_waller = param == 3;
        sf::fit_exv_debye_waller = param == 4;
        SimpleDataset data(std::vector<double>(q, q + n), std::vector<double>(I, I + n),
                           std::vector<double>(sigma, sigma + n));
        std::unique_ptr<hist::DistanceHistogram> h = std::move(static_cast<Result*>(r)->h);
        fitter::SmartFitter f(data, std::move(h));
        const auto t0 = std::chrono::steady_clock::now();
        auto res = f.fit();
        out[5] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        // the inner linear fit's a and b are added in front of the fitted parameter
        const auto v = res->get_parameter_values();
        out[0] = v.back();
        out[1] = double(res->get_parameter("a"));
        out[2] = double(res->get_parameter("b"));
        out[3] = res->fval;
        out[4] = res->fevals;
        sf::fit_hydration = true;  // the defaults (FitSettings.cpp:12-16)
        sf::fit_excluded_volume = sf::fit_solvent_density = sf::fit_atomic_debye_waller = sf::fit_exv_debye_waller = false;
    });
}

// hist::distance_calculator::SimpleCalculator<true, false> on a job list over point sets {x, y, z, w}
// (set s is rows [set_off[s], set_off[s+1]) of pts): job k is enqueue_calculate_self(set ja[k],
// scaling[k], merge[k]) when jb[k] < 0, else enqueue_calculate_cross(set ja[k], set jb[k], ...).
// Results: the self merge ids, then the cross merge ids, each ascending; keys[2 r] = is_cross,
// keys[2 r + 1] = merge id; out[(3 r + {0, 1, 2}) * bin_count + i] = value, count, bin-centre sum.
int ref_calculator(const double* pts, const int* set_off, int n_sets, int n_jobs, const int* ja, const int* jb,
                   const int* scaling, const int* merge, int* n_results, int* keys, double* out) {
    return guarded([&] {
        if (custom_width()) run_calculator<true>(pts, set_off, n_sets, n_jobs, ja, jb, scaling, merge, n_results, keys, out);
        else run_calculator<false>(pts, set_off, n_sets, n_jobs, ja, jb, scaling, merge, n_results, keys, out);
    });
}

// hist::exact_debye_transform (source/core/hist/intensity_calculator/ExactDebyeCalculator.cpp:13-58).
int ref_exact_debye(void* m, const double* q, int nq, double* Iq) {
    return guarded([&] {
        std::vector<double> qv(q, q + nq);
        auto I = hist::exact_debye_transform(*static_cast<FixedVolumeMolecule*>(m), qv);
        std::memcpy(Iq, I.data(), I.size() * sizeof(double));
    });
}

// fitter::detail::LinearLeastSquares::fit (source/core/fitter/detail/LinearLeastSquares.cpp:26-55):
// out = {a, b, sigma_a, sigma_b, chi2}.
int ref_linear_lsq(const double* data, const double* model, const double* err, int n, double* out) {
    return guarded([&] {
        std::vector<double> d(data, data + n), m(model, model + n), e(err, err + n);
        fitter::detail::LinearLeastSquares f(d, m, e);
        auto r = f.fit();
        out[0] = r->get_parameter(0u).value;
        out[1] = r->get_parameter(1u).value;
        out[2] = r->get_parameter(0u).error.max;
        out[3] = r->get_parameter(1u).error.max;
        out[4] = r->fval;
    });
}

}  // extern "C"
