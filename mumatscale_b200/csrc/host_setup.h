// host_setup.h — host-side state and setup of the nucleation sites.
//
// The reference draws its nucleation sites and orientations from glibc
// rand() streams, one per MPI rank (srand(rank+1+seed), ca_main.c:215), in a
// fixed order during setup and at grain activation.  These draws define the
// result, so they are replayed here exactly, on the host, per emulated rank.
#pragma once

#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mms_internal.h"

namespace mms {

// One emulated MPI rank: its rand() stream (srand(rank+1+seed),
// ca_main.c:215) and its list of deck-defined nucleation points (nuc_pt).
struct NucPt {  // nucleation_t, globals.h:147-160
    double x, y, z;
    size_t cx, cy, cz;
    double gx, gy, gz;
    double threshold;
};

// A copy of one rand() stream's position (the random_r state holds pointers
// into its own buffer, so copies rebase them).
struct RngState {
    struct random_data rd;
    char state[128];
    long ncalls = 0;
    int have_gauss = 0;
    float gauss_next = 0.f;
};

struct Rank {
    struct random_data rd;
    char state[128];
    unsigned seed = 0;
    long ncalls = 0;
    long ncalls_presb = 0;  // calls made before init_sb_nucleation
    int have_gauss = 0;
    float gauss_next = 0.f;
    int sbx = 0, sby = 0, sbz = 0;
    std::vector<NucPt> nuc;
    std::vector<std::array<double, 3>> angles;  // orientation draws after setup
    long long rng_base = 0;                     // draw number of device table entry 0

    void seed_with(unsigned s);
    void save(RngState &out) const;
    void restore(const RngState &in);
    int32_t rand_();
    // getRandScale, functions.c:440-445
    float scale();
    // getRandomGaussian, functions.c:376-406
    float gauss();
};

// nucleate_grain's rotation matrix (grain.c:314-336), row-major
void rotmat_from_angles(double a0, double a1, double a2, double *R);

// realcoord2scoord (functions.c:91-107) and CELLCOORD2REALCOORDn
// (functions.h:284-286)
void real2cell(const mms_params &p, double x, double y, double z, size_t *i, size_t *j, size_t *k);
double cell2real(const mms_params &p, int axis, double i);
// setNucOrientation (grain.c:117-130)
void draw_orientation(const mms_params &p, Rank &r, NucPt &n);

// Geometry of the global halo'd grid for a parameter set.
Geo make_geo(const mms_params &p);
// Mold flags: pad faces of the global halo (tempPrepareSB_int, temperature.c:199-214).
std::vector<signed char> make_mold(const Geo &g);
// Seeds every emulated rank (ca_main.c:215) and assigns its subblock.
void init_ranks(const mms_params &p, const Geo &g, std::vector<Rank> &ranks);
// init_nucleation_sites (grain.c:602-713, rank 0): the deck's FixedNuc and
// NucVolume points (rank 0 draws the latter), distributed to their ranks.
void assign_deck_sites(const mms_params &p, const Geo &g, const std::vector<mms_fixed_nuc> &fixed,
                       const std::vector<mms_nuc_volume> &vols, std::vector<Rank> &ranks);
// init_nucleation_sites (grain.c:602-713, rank 0) and init_sb_nucleation
// (grain.c:930-1010, every rank): fills the dense threshold array (+inf where
// no site) and each rank's deck-defined nucleation points.
void setup_sites(const mms_params &p, const Geo &g, const std::vector<mms_fixed_nuc> &fixed,
                 const std::vector<mms_nuc_volume> &vols, std::vector<Rank> &ranks, std::vector<float> &thr,
                 const std::vector<signed char> &mold);

}  // namespace mms
