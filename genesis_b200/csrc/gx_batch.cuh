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
                                   // 3 persistent cooperative launch of the all-replica phases
    gx::BatchFlat* flat = nullptr;  // state of mode 2
};

namespace gx {
int batch_flat_step(gx_batch* b, int nsteps, uint64_t* launches);
int batch_coop_step(gx_batch* b, int nsteps, uint64_t* launches);
}
