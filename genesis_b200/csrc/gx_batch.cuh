// gx_batch.cuh -- state of a gx_batch (many small universes advanced
// together), shared by the persistent one-CTA-per-replica launch
// (gx_batch.cu) and the all-replica graph of kernels (gx_batch_flat.cu).
#pragma once

#include <string>
#include <vector>

#include "gx_pair_f32.cuh"

namespace gx {

constexpr int kBThreads = 512;
constexpr uint32_t kBMaxCells = 4096;  // cells per replica held in shared memory

struct RepDesc {
    GridGeom g;
    uint32_t base, n;
    double half_box[3];
    double target, tau;
    int thermo;
};

struct BatchArrays {
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *mass, *inv_mass;
    uint8_t* kind;
    uint32_t *key, *idx, *skey;
    float4* pos4;
    long long* F;  // 3 * total, SoA
    size_t total;
};

struct BatchParams {
    double dt, half_dt, k_thermal;
    int boundaries, nsteps;
};

LawF32 make_law32(const gx_handle* h);

struct BatchFlat;  // gx_batch_flat.cu
void batch_flat_free(BatchFlat* f);
struct BatchNl;  // gx_batch_nl.cu
void batch_nl_free(BatchNl* n);
// A replica's atom range (concatenated order) and its Berendsen thermostat.
struct RepThermo {
    uint32_t base, n;
    double target, tau;
    int thermo;
};

}  // namespace gx

struct gx_batch {
    gx_params p;
    gx::LawF32 L;
    int nrep = 0;
    std::vector<gx::RepDesc> reps;
    gx::RepDesc* d_reps = nullptr;
    int* d_order = nullptr;
    gx::BatchArrays A{};
    size_t total = 0;
    gx::PairF* d_tab = nullptr;
    double* d_out = nullptr;
    uint32_t* d_err = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {};
    std::string err;
    double pair_sigma[gx::kNElem * gx::kNElem], pair_eps[gx::kNElem * gx::kNElem];
    bool has_state = false;
    int mode = 2;                  // 1 persistent launch (a CTA per replica), 2 all-replica graph,
                                   // 3 persistent cooperative launch of the all-replica phases,
                                   // 4 all-replica graph over persistent neighbour lists
    gx::BatchFlat* flat = nullptr;  // state of modes 2-4
    gx::BatchNl* nl = nullptr;      // lists of mode 4
    double rc = 0.0;                // pair cutoff
    double nl_skin = -1.0;          // mode 4 list skin (< 0: 0.1 rc)
    uint64_t version = 0;           // bumped whenever the state changes other than by a mode-4 step
};

namespace gx {
int batch_flat_step(gx_batch* b, int nsteps, uint64_t* launches);
int batch_coop_step(gx_batch* b, int nsteps, uint64_t* launches);
int batch_nl_step(gx_batch* b, int nsteps, uint64_t* launches);
bool batch_nl_eligible(const gx_batch* b);  // every replica: >= 3 list cells per axis, >= 128 atoms
int batch_nl_rebuilds(gx_batch* b, uint64_t* out);
int batch_nl_stats(gx_batch* b, uint64_t* entries, uint64_t* overflowed);
// shared with mode 4 (gx_batch_flat.cu): prepares the all-replica tables and
// returns them; the end-of-step commit of the pending scales
struct FlatShared {
    const uint32_t* rep_of;
    const RepThermo* th;
    double* lam;
    unsigned long long* acc;
};
int flat_shared(gx_batch* b, FlatShared* out);
void flat_commit(gx_batch* b, gx_handle* h);
}
