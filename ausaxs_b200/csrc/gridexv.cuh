// Grid excluded-volume dummies and grid volume on the device (see gridexv.cu).
#pragma once
#include "engine.cuh"

namespace ausaxs_b200 {

struct GridExv {
    DevBuf work;        // the cell grid and compaction counters
    DevBuf points;      // dummies: float4 {x, y, z, EXCLUDED_VOLUME}
    long long count = 0;
    double volume = 0;  // A^3 (kept cells x 1 A^3): Molecule::get_volume_grid()
    // atoms / waters: device records ({x, y, z, ff} / {x, y, z, w}); lo/hi: their bounding box.
    // Writes the dummies into `out` when it is non-null and holds `cap` >= count records, else into
    // `points` when want_points.  Synchronises once (the dummy count).
    void run(Ctx& C, const float4* atoms, int na, const float4* waters, int nw, const float lo[3], const float hi[3],
             bool want_points, float4* out = nullptr, long long cap = 0);
};

}  // namespace ausaxs_b200
