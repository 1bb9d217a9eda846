// Hydration shell on the device (see hydrate.cu).
#pragma once
#include "engine.cuh"

namespace ausaxs_b200 {

constexpr int kHydDirections = 26;  // RadialHydration::prepare_rotations(8): unique unit vectors

// Grid(bodies)'s axes over the atoms alone (Grid.cpp:34-102): gmin[3], bins[3].
void hydrate_axes(const double* xyz, long long n, double gmin[3], int bins[3]);

// The atom state of a hydration grid's cells (one byte per cell, the reference's A_CENTER / A_AREA /
// VOLUME bits): Grid::add of atoms with their expansion, and Grid::remove of atoms at their current
// positions.  Enqueued on the context's stream; *err is set when an atom lies outside the grid.
void hydration_cells_check(const double gmin[3], const int bins[3]);
void hydration_add(Ctx& C, uint8_t* cells, const double gmin[3], const int bins[3], const double* atoms, const int32_t* ff,
                   long long n, int* err);
void hydration_remove(Ctx& C, uint8_t* cells, const double gmin[3], const int bins[3], const double* atoms,
                      const int32_t* ff, long long n, int* err);

struct Hydrator {
    DevBuf in;      // atoms (double, n x 3), form-factor types, noise table
    DevBuf cells;   // cell states of one-shot calls
    DevBuf keys;    // [3][key_cells] epoch-tagged minimum candidate indices (accepted, two undecided)
    size_t key_cells = 0;
    DevBuf list;    // candidates that survive the static tests, in candidate order, and their state
    DevBuf work;    // block counts, round counters, output staging
    uint32_t call_epoch = 0, round_epoch = 0;
    long long count = 0;   // waters
    long long survivors = 0;
    int rounds = 0;
    // RadialHydration over the grid `cells` (device): atoms (device, n x 3 doubles) in visiting order,
    // ff their form-factor types; noise: device table (n x 26 x 3) or null, then seed != 0 draws
    // Gaussian noise (sigma 0.75 A) per candidate.  Leaves the waters (double, count x 3) and their
    // candidate indices (int64) at waters() / candidates().  Synchronises once per batch of rounds
    // and once for the count.
    void generate(Ctx& C, const uint8_t* cells, const double gmin[3], const int bins[3], const double* atoms,
                  const int32_t* ff, long long n, const double* noise, unsigned long long seed);
    // a fresh grid of these atoms, then generate
    void run(Ctx& C, const double* atoms, const int32_t* ff, long long n, const double gmin[3], const int bins[3],
             const double* noise, unsigned long long seed);
    const double* waters() const { return work.as<double>(off_waters); }
    const long long* candidates() const { return work.as<long long>(off_cands); }

  private:
    size_t off_waters = 0, off_cands = 0;
};

}  // namespace ausaxs_b200
