// sites.h — nucleation sites drawn on the device (sites.cu).
#pragma once

#include <string>
#include <vector>

namespace mms {

struct SiteDrawArgs {
    long long total;                 // cells to visit: this context's ranks' cells
    long long qbase;                 // list position of the first (first rank x sbcells)
    long long sbcells;               // cells per subblock
    int sbx, sby, sbz, nsbx, nsby;   // NCellsPerSB, NSubblocks x and y
    long long gx, gy, gz;            // whole domain's interior cells
    int padx, pady, padz;            // pad (mold) faces of the whole domain
    int rank0;                       // first emulated rank of this context
    long long kz0;                   // this context's z offset in the whole domain
    long long dsy, dsz;              // this context's device strides
    unsigned seed;                   // RandSeedVal
    double vol_centre, vol_sigma, surf_centre, surf_sigma;
    long long npreset;               // set by site_draw_device
};

// The site list in (rank, local raster) order: device cell index,
// threshold, rank relative to rank0.  pv, ps: per rank of the whole
// domain, the volume and surface selection probabilities; presets: list
// positions (sorted) and thresholds of deck-defined sites.  Returns 0, or 1
// with err set.
int site_draw_device(const SiteDrawArgs &args, const std::vector<double> &pv, const std::vector<double> &ps,
                     const std::vector<long long> &preset_q, const std::vector<float> &preset_thr,
                     std::vector<long long> &cells, std::vector<float> &thr, std::vector<int> &rank, std::string &err);

}  // namespace mms
