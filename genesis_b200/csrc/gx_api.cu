// gx_api.cu -- C ABI: handle lifecycle, state transfer, the force-schedule
// systems and the fused tick.  Declarations and the reference interface each
// entry point replaces are in include/genesis_gpu.h.
#include <cmath>
#include <cstring>
#include <string>

#include "gx_internal.cuh"

namespace gx {
int upload_pair_table_f64(gx_handle* h);
size_t red_doubles(size_t cap);
}  // namespace gx

namespace gx {

int set_err(gx_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}
int cuda_err(gx_handle* h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return set_err(h, GX_ERR_CUDA, m);
}

static const int kAllOffsets[27][3] = {  // src/physics/grid.rs:37-47
    {-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, -1}, {-1, 0, 0}, {-1, 0, 1}, {-1, 1, -1}, {-1, 1, 0}, {-1, 1, 1},
    {0, -1, -1},  {0, -1, 0},  {0, -1, 1},  {0, 0, -1},  {0, 0, 0},  {0, 0, 1},  {0, 1, -1},  {0, 1, 0},  {0, 1, 1},
    {1, -1, -1},  {1, -1, 0},  {1, -1, 1},  {1, 0, -1},  {1, 0, 0},  {1, 0, 1},  {1, 1, -1},  {1, 1, 0},  {1, 1, 1}};

GridGeom make_grid(const double box[3], double min_cell, int* ok) {
    GridGeom g;
    std::memset(&g, 0, sizeof g);
    *ok = 0;
    if (!(min_cell > 0.0) || !std::isfinite(min_cell)) return g;
    double total = 1.0;
    for (int k = 0; k < 3; ++k) {
        if (!(box[k] > 0.0) || !std::isfinite(box[k])) return g;
        double c = std::floor(box[k] / min_cell);  // grid.rs:68
        if (c < 1.0) c = 1.0;
        if (c > 1048576.0) return g;
        g.n[k] = (uint32_t)c;
        total *= c;
    }
    if (total > 268435456.0) return g;
    g.ncell = g.n[0] * g.n[1] * g.n[2];
    for (int k = 0; k < 3; ++k) {
        g.L[k] = box[k];
        g.cell[k] = box[k] / (double)g.n[k];
        g.cellf[k] = (float)g.cell[k];
        g.Lf[k] = (float)box[k];
        g.invLf[k] = (float)(1.0 / box[k]);
        if (g.n[k] < 3) g.minimg_mask |= 1 << k;
    }
    // Canonical offsets (grid.rs:275-296): zero on degenerate axes, first
    // nonzero component +1.  Kept in ALL_OFFSETS order.
    g.nhalf = 0;
    for (const auto& o : kAllOffsets) {
        if (o[0] == 0 && o[1] == 0 && o[2] == 0) continue;
        bool degen_nonzero = false;
        for (int k = 0; k < 3; ++k)
            if (g.n[k] <= 1 && o[k] != 0) degen_nonzero = true;
        if (degen_nonzero) continue;
        int first = o[0] != 0 ? o[0] : (o[1] != 0 ? o[1] : o[2]);
        if (first != 1) continue;
        for (int k = 0; k < 3; ++k) g.half[g.nhalf][k] = (int8_t)o[k];
        ++g.nhalf;
    }
    g.nfull = 2 * g.nhalf;
    for (int q = 0; q < g.nhalf; ++q)
        for (int k = 0; k < 3; ++k) {
            g.full[q][k] = g.half[q][k];
            g.full[g.nhalf + q][k] = (int8_t)-g.half[q][k];
        }
    *ok = 1;
    return g;
}

// The pair pass's events of gx_set_pass_timing ("force_*" slots): recorded
// in eager ticks, and inside a capture as external event nodes of the
// tick's graph, so that a replayed tick times its own pass.
void pass_mark(gx_handle* h, const char* name, int k) {
    if (!h->pass_timing || std::strncmp(name, "force_", 6) != 0) return;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &st) != cudaSuccess) return;
    cudaEventRecordWithFlags(h->pass_ev[k], h->stream,
                             st == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault);
}

void prof_begin(gx_handle* h, const char* name) {
    pass_mark(h, name, 0);
    if (!h->prof_on) return;
    ProfSlot* s = nullptr;
    for (auto& p : h->prof)
        if (p.name == name || std::strcmp(p.name, name) == 0) s = &p;
    if (!s) {
        h->prof.push_back(ProfSlot{name, 0, 0.0, {}});
        s = &h->prof.back();
    }
    cudaEvent_t a, b;
    if (h->ev_pool.size() >= 2) {
        a = h->ev_pool.back();
        h->ev_pool.pop_back();
        b = h->ev_pool.back();
        h->ev_pool.pop_back();
    } else {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    cudaEventRecord(a, h->stream);
    s->ev.push_back(a);
    s->ev.push_back(b);
}
void prof_end(gx_handle* h, const char* name) {
    pass_mark(h, name, 1);
    if (!h->prof_on) return;
    for (auto& p : h->prof)
        if (p.name == name || std::strcmp(p.name, name) == 0) {
            cudaEventRecord(p.ev.back(), h->stream);
            p.launches += 1;
            return;
        }
}

}  // namespace gx

using namespace gx;

namespace {

const double kElementMass[kNElem] = {1.008, 4.0026, 12.011, 14.007, 15.999,
                                     22.99, 28.085, 30.974, 32.06,  55.845};  // atom_type.rs:80-93

void free_buf(StateBuf& b) {
    cudaFree(b.x);
    cudaFree(b.vx);
    cudaFree(b.ax);
    cudaFree(b.charge);
    cudaFree(b.elem);
    cudaFree(b.slot);
    std::memset(&b, 0, sizeof b);
}

int alloc_buf(gx_handle* h, StateBuf& b, size_t cap) {
    free_buf(b);
    GX_CUDA(h, cudaMalloc(&b.x, 3 * cap * sizeof(double)));
    GX_CUDA(h, cudaMalloc(&b.vx, 3 * cap * sizeof(double)));
    GX_CUDA(h, cudaMalloc(&b.ax, 3 * cap * sizeof(double)));
    GX_CUDA(h, cudaMalloc(&b.charge, 3 * cap * sizeof(double)));
    GX_CUDA(h, cudaMalloc(&b.elem, 2 * cap));
    GX_CUDA(h, cudaMalloc(&b.slot, cap * sizeof(uint32_t)));
    b.y = b.x + cap;
    b.z = b.x + 2 * cap;
    b.vy = b.vx + cap;
    b.vz = b.vx + 2 * cap;
    b.ay = b.ax + cap;
    b.az = b.ax + 2 * cap;
    b.mass = b.charge + cap;
    b.inv_mass = b.charge + 2 * cap;
    b.kind = b.elem + cap;
    return GX_OK;
}

int ensure_capacity(gx_handle* h, size_t n) {
    if (n <= h->cap && h->cap) return GX_OK;
    size_t cap = n < 1024 ? 1024 : n;
    for (int k = 0; k < 2; ++k) {
        int rc = alloc_buf(h, h->buf[k], cap);
        if (rc) return rc;
    }
    cudaFree(h->key);
    cudaFree(h->pos4);
    cudaFree(h->F);
    cudaFree(h->host_stage);
    cudaFree(h->red);
    GX_CUDA(h, cudaMalloc(&h->key, 5 * cap * sizeof(uint32_t)));
    h->key_sorted = h->key + cap;
    h->perm = h->key + 2 * cap;
    h->pos_of_slot = h->key + 3 * cap;
    h->entity = h->key + 4 * cap;
    GX_CUDA(h, cudaMalloc(&h->pos4, cap * sizeof(float4)));
    GX_CUDA(h, cudaMalloc(&h->F, 3 * cap * sizeof(long long)));
    GX_CUDA(h, cudaMalloc(&h->host_stage, 3 * cap * sizeof(double) + cap * sizeof(uint32_t)));
    h->u8_stage = (uint8_t*)(h->host_stage + 3 * cap);
    GX_CUDA(h, cudaMalloc(&h->red, red_doubles(cap) * sizeof(double)));
    h->cap = cap;
    int rc = upload_pair_table_f64(h);
    if (rc) return rc;
    return GX_OK;
}

__global__ void k_aos_to_soa(const double* __restrict__ aos, double* x, double* y, double* z, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = aos[3 * i];
    y[i] = aos[3 * i + 1];
    z[i] = aos[3 * i + 2];
}
// sorted SoA -> slot-ordered AoS
__global__ void k_soa_to_aos(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                             const uint32_t* __restrict__ slot, double* __restrict__ aos, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s = slot[i];
    aos[3 * s] = x[i];
    aos[3 * s + 1] = y[i];
    aos[3 * s + 2] = z[i];
}
// slot-ordered AoS -> sorted SoA (per-tick host column sync)
__global__ void k_aos_to_sorted(const double* __restrict__ aos, const uint32_t* __restrict__ pos_of_slot, double* x,
                                double* y, double* z, uint32_t n) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t p = pos_of_slot[s];
    x[p] = aos[3 * s];
    y[p] = aos[3 * s + 1];
    z[p] = aos[3 * s + 2];
}
// Eight independent FMA chains per thread (diagnostic FP32 peak probe).
__global__ void k_fma_peak(float* out, int iters, float seed) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + 1e-3f * (threadIdx.x + k);
    const float m = 0.9999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}
__global__ void k_fma_peak_f64(double* out, int iters, double seed) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + 1e-3 * (threadIdx.x + k);
    const double m = 0.9999999999, c = 1e-12;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678) out[threadIdx.x] = s;  // keeps the chains live
}
__global__ void k_init_slots(StateBuf b, uint32_t* pos_of_slot, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    b.slot[i] = i;
    pos_of_slot[i] = i;
    b.inv_mass[i] = xdiv(1.0, b.mass[i]);  // the 1.0 / mass of systems/forces.rs:339
}
__global__ void k_fill_d(double* p, uint32_t n, double v) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
// Appends this tick's observables at record index dcount[5] (a device-side
// cursor, so the same launch sequence can be replayed from a CUDA graph).
// One tick's record.  `scale`: dscal[1] and dscal[4] hold K and the speed
// sum before the thermostat's scale lambda = dscal[0]; the record takes
// those of lambda v, lambda^2 K and lambda S (equal to the sums over the
// scaled components up to the rounding of the products, ~1e-16 relative).
__global__ void k_record(gx_tick_stats* rec, const double* dscal, unsigned long long* dcount, int thermo,
                         int scale) {
    unsigned long long k = dcount[5];
    const double l = scale ? dscal[0] : 1.0;
    rec[k].kinetic = scale ? xmul(xmul(dscal[1], l), l) : dscal[1];
    rec[k].speed_sum = scale ? xmul(dscal[4], l) : dscal[4];
    rec[k].potential = dscal[2];
    rec[k].bond_energy = dscal[3];
    rec[k].lambda = thermo ? dscal[0] : 1.0;
    rec[k].pairs = dcount[0];
    dcount[5] = k + 1;
}

// The speed partials summed as k_finalize_sum sums them (the same order, so
// the same value) into dscal[4], then the record of k_record: one launch for
// both on the list path's recorded ticks.
constexpr int kRecThreads = 256;
__global__ void __launch_bounds__(kRecThreads) k_record_sum(const double* __restrict__ spart, int nb,
                                                            gx_tick_stats* rec, double* dscal,
                                                            unsigned long long* dcount, int thermo, int scale) {
    __shared__ double sh[kRecThreads / 32];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += kRecThreads) v = xadd(v, spart[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < kRecThreads / 32) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    if (threadIdx.x != 0) return;
    dscal[4] = v;
    unsigned long long k = dcount[5];
    const double l = scale ? dscal[0] : 1.0;
    rec[k].kinetic = scale ? xmul(xmul(dscal[1], l), l) : dscal[1];
    rec[k].speed_sum = scale ? xmul(v, l) : v;
    rec[k].potential = dscal[2];
    rec[k].bond_energy = dscal[3];
    rec[k].lambda = thermo ? dscal[0] : 1.0;
    rec[k].pairs = dcount[0];
    dcount[5] = k + 1;
}

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

void invalidate_graphs(gx_handle* h) {
    for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 2; ++b) {
            if (h->graph_exec[a][b]) cudaGraphExecDestroy(h->graph_exec[a][b]);
            h->graph_exec[a][b] = nullptr;
            h->graph_key[a][b] = 0;
        }
        if (h->graph_multi[a]) cudaGraphExecDestroy(h->graph_multi[a]);
        h->graph_multi[a] = nullptr;
        h->graph_multi_key[a] = 0;
    }
}

// Ticks of the list path captured into one graph when a step call has that
// many left: fewer graph launches for small systems, whose ticks last only
// tens of microseconds.
constexpr int kTicksPerGraph = 8;

// The pending Berendsen scale is folded into the next kernel that reads v;
// anything else that reads v first commits it.
int commit_lambda(gx_handle* h) {
    if (!h->lambda_pending) return GX_OK;
    launch_apply_lambda(h, h->buf[h->cur], (uint32_t)h->n, h->dscal + 0);
    h->lambda_pending = false;
    return GX_OK;
}

// The device error word of the pair pass as a status (and cleared).
int step_error(gx_handle* h, uint32_t e) {
    if (!e) return GX_OK;
    cudaMemset(h->derr, 0, sizeof(uint32_t));
    if (e & kErrNonFinite) return set_err(h, GX_ERR_NONFINITE, "non-finite force in the pair pass");
    if (e & kErrSaturation) return set_err(h, GX_ERR_SATURATION, "fixed-point force saturated");
    if (e & kErrTimeout) return set_err(h, GX_ERR_TIMEOUT, "shared-memory staging wait timed out");
    return set_err(h, GX_ERR_CUDA, "unknown device error");
}

}  // namespace

namespace gx {
int commit_pending_lambda(gx_handle* h) { return commit_lambda(h); }
int take_step_errors(gx_handle* h) {
    if (!h->step_errs_pending) return GX_OK;
    h->step_errs_pending = false;
    return step_error(h, *h->herr);
}
int settle_step_errors(gx_handle* h) {
    if (!h->step_errs_pending) return GX_OK;
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    return take_step_errors(h);
}
}  // namespace gx

namespace {

int require_state(gx_handle* h) {
    if (!h) return GX_ERR_ARG;
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    return GX_OK;
}

// Cell list of the force grid: keys, counting sort, reorder (double buffer).
int rebuild_cells(gx_handle* h) {
    uint32_t n = (uint32_t)h->n;
    StateBuf& src = h->buf[h->cur];
    launch_cell_keys(h, h->fgrid, src, n, h->key);
    int rc = counting_sort(h, h->cl, h->fgrid.ncell, h->key, n, h->perm);
    if (rc) return rc;
    launch_gather(h, src, h->buf[h->cur ^ 1], h->perm, h->key, h->key_sorted, n, h->pos_of_slot);
    h->cur ^= 1;
    h->sorted = true;
    h->nl_valid = false;
    if (h->precision == GX_MIXED) launch_build_pos4(h, h->fgrid, h->buf[h->cur], h->key_sorted, n, h->pos4);
    return GX_OK;
}

int check_kinds(gx_handle* h) {
    if (h->precision == GX_MIXED && h->nkinds > kMaxKinds)
        return set_err(h, GX_ERR_UNSUPPORTED,
                       "mixed precision supports at most 16 distinct (element, charge) kinds, (element, charge, mass) "
                       "with gravity");
    return GX_OK;
}

int upload_pairf(gx_handle* h) {
    if (!h->d_pairf) GX_CUDA(h, cudaMalloc(&h->d_pairf, kMaxKinds * kMaxKinds * sizeof(PairF)));
    PairF tab[kMaxKinds * kMaxKinds];
    std::memset(tab, 0, sizeof tab);
    int nk = h->nkinds < kMaxKinds ? h->nkinds : kMaxKinds;
    for (int a = 0; a < nk; ++a)
        for (int b = 0; b < nk; ++b) {
            int ea = h->kind_elem[a], eb = h->kind_elem[b];
            double sg = h->fs.pair_sigma[ea * kNElem + eb], ep = h->fs.pair_eps[ea * kNElem + eb];
            PairF& t = tab[a * nk + b];
            t.sigma = (float)sg;
            t.half_sigma = (float)(0.5 * sg);
            t.inv_half_sigma = (float)(2.0 / sg);
            t.eps4 = (float)(4.0 * ep);
            t.eps24 = (float)(24.0 * ep);
            // symmetric by construction: (i, j) and (j, i) must round identically
            int lo = a < b ? a : b, hi = a < b ? b : a;
            t.qq = (float)(h->p.coulomb_constant * h->kind_charge[lo] * h->kind_charge[hi]);
            t.gm = (float)(h->p.gravity_constant * h->kind_mass[lo] * h->kind_mass[hi]);
        }
    GX_CUDA(h, cudaMemcpy(h->d_pairf, tab, sizeof tab, cudaMemcpyHostToDevice));
    return GX_OK;
}

}  // namespace

extern "C" {

const char* gx_status_string(int s) {
    switch (s) {
        case GX_OK: return "ok";
        case GX_ERR_ARG: return "invalid argument";
        case GX_ERR_OOM: return "device allocation failed";
        case GX_ERR_CUDA: return "CUDA error";
        case GX_ERR_CAPACITY: return "capacity exceeded";
        case GX_ERR_SATURATION: return "fixed-point saturation";
        case GX_ERR_NONFINITE: return "non-finite value";
        case GX_ERR_TIMEOUT: return "device wait timed out";
        case GX_ERR_UNSUPPORTED: return "unsupported configuration";
        case GX_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

const char* gx_last_error(const gx_handle* h) { return h ? h->err.c_str() : "null handle"; }

int gx_create(const gx_params* p, gx_handle** out) {
    if (!p || !out) return GX_ERR_ARG;
    *out = nullptr;
    if (p->precision != GX_FP64 && p->precision != GX_MIXED) return GX_ERR_ARG;
    if (!(p->dt == p->dt) || !(p->thermal_constant == p->thermal_constant)) return GX_ERR_ARG;
    gx_handle* h = new gx_handle();
    h->p = *p;
    h->precision = p->precision;
    // ForceSystem::new (systems/forces.rs:100-142) and LjTable::new (physics/forces.rs:223-237).
    ForceSetup& fs = h->fs;
    double max_pair = 0.0, max_sigma = 0.0;
    for (int i = 0; i < kNElem; ++i) {
        max_sigma = std::fmax(max_sigma, p->sigma[i]);
        for (int j = 0; j < kNElem; ++j) {
            double s = 0.5 * (p->sigma[i] + p->sigma[j]);
            double e = p->thermal_constant * std::sqrt(p->epsilon_k[i] * p->epsilon_k[j]);
            max_pair = std::fmax(max_pair, s);
            fs.pair_sigma[i * kNElem + j] = s;
            fs.pair_eps[i * kNElem + j] = e;
        }
    }
    fs.lj_rc = std::fmax(p->lj_cutoff_factor, 1.0) * max_pair;
    fs.lj_ron = 0.9 * fs.lj_rc;
    fs.coul_rc = p->enable_electrostatics ? std::fmax(p->coulomb_cutoff, 1.0) * max_sigma : 0.0;
    fs.grav_rc = p->enable_gravity ? std::fmax(p->gravity_cutoff, 1.0) * max_sigma : 0.0;
    fs.rc = std::fmax(std::fmax(fs.lj_rc, fs.coul_rc), fs.grav_rc);
    fs.coul_ron = 0.9 * fs.coul_rc;
    fs.grav_ron = 0.9 * fs.grav_rc;
    fs.bond_k_bind = p->bond_k_bind;
    fs.max_sigma = max_sigma;
    fs.r_eq_factor = std::pow(2.0, 1.0 / 6.0);
    fs.curv_factor = 72.0 * std::pow(2.0, -1.0 / 3.0);
    int ok = 0;
    h->fgrid = make_grid(p->box, fs.rc, &ok);
    if (!ok) {
        int rc = set_err(h, GX_ERR_ARG, "invalid box or cutoff (grid would be empty or too large)");
        *out = h;
        return rc;
    }
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&h->dscal, 16 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&h->dcount, 16 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&h->derr, sizeof(uint32_t));
    if (e != cudaSuccess) {
        int rc = cuda_err(h, e, "gx_create");
        *out = h;
        return rc;
    }
    double init[16] = {1.0, 0, 0, 0, 0, 1.0};
    cudaMemcpy(h->dscal, init, sizeof init, cudaMemcpyHostToDevice);
    cudaMemset(h->dcount, 0, 16 * sizeof(unsigned long long));
    cudaMemset(h->derr, 0, sizeof(uint32_t));
    *out = h;
    return GX_OK;
}

void gx_destroy(gx_handle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    invalidate_graphs(h);
    adjoint_free(h);
    nl_free(h);
    tracker_free(h);
    lens_free(h);
    collide_free(h);
    export_free(h);
    snapshot_free(h);
    for (cudaEvent_t e : h->pass_ev)
        if (e) cudaEventDestroy(e);
    if (h->io_stream) {
        cudaStreamSynchronize(h->io_stream);
        cudaStreamDestroy(h->io_stream);
    }
    for (cudaEvent_t e : h->io_ev)
        if (e) cudaEventDestroy(e);
    cudaFree(h->io_stage);
    if (h->herr) cudaFreeHost(h->herr);
    free_buf(h->buf[0]);
    free_buf(h->buf[1]);
    cudaFree(h->key);
    cudaFree(h->pos4);
    cudaFree(h->F);
    cudaFree(h->host_stage);
    cudaFree(h->red);
    cudaFree(h->dscal);
    cudaFree(h->dcount);
    cudaFree(h->derr);
    cudaFree(h->d_pairf);
    cudaFree(h->bonds);
    cells_free(h->cl);
    for (auto& s : h->prof)
        for (auto ev : s.ev) cudaEventDestroy(ev);
    for (auto ev : h->ev_pool) cudaEventDestroy(ev);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int gx_set_precision(gx_handle* h, int precision) {
    if (!h || (precision != GX_FP64 && precision != GX_MIXED)) return GX_ERR_ARG;
    h->precision = precision;
    h->sorted = false;
    invalidate_graphs(h);
    return check_kinds(h);
}

size_t gx_num_atoms(const gx_handle* h) { return h ? h->n : 0; }

int gx_set_state(gx_handle* h, size_t n, const double* pos, const double* vel, const double* acc,
                 const uint8_t* elem, const double* charge, const double* mass, const uint32_t* entity) {
    if (!h || (n && (!pos || !vel || !elem))) return GX_ERR_ARG;
    if (n > 0x7FFFFFFFu) return set_err(h, GX_ERR_ARG, "too many atoms");
    for (size_t i = 0; i < n; ++i)
        if (elem[i] >= kNElem) return set_err(h, GX_ERR_ARG, "element index out of range (0..9)");
    GX_CUDA(h, cudaSetDevice(h->p.device));
    int rc = ensure_capacity(h, n);
    if (rc) return rc;
    h->n = n;
    h->cur = 0;
    h->sorted = false;
    h->nl_valid = false;
    h->nl_fresh = false;
    tracker_free(h);  // new atoms: the open episodes no longer apply
    h->lambda_pending = false;
    invalidate_graphs(h);
    h->nbonds = 0;  // bonds name slots of the previous atoms
    GX_CUDA(h, cudaMemsetAsync(dnbonds(h), 0, sizeof(unsigned long long), h->stream));
    StateBuf& b = h->buf[0];
    uint32_t un = (uint32_t)n;
    std::vector<double> tmp(n);
    // kinds: distinct (element, charge) pairs -- with gravity (element,
    // charge, mass) -- in first-seen order
    h->nkinds = 0;
    std::vector<uint8_t> kind(n);
    const bool by_mass = h->p.enable_gravity != 0;
    for (size_t i = 0; i < n; ++i) {
        double q = charge ? charge[i] : h->p.charge[elem[i]];
        double m = by_mass ? (mass ? mass[i] : kElementMass[elem[i]]) : 0.0;
        int found = -1;
        for (int k = 0; k < h->nkinds && k < kMaxKinds; ++k)
            if (h->kind_elem[k] == elem[i] && h->kind_charge[k] == q && h->kind_mass[k] == m) found = k;
        if (found < 0) {
            if (h->nkinds < kMaxKinds) {
                h->kind_elem[h->nkinds] = elem[i];
                h->kind_charge[h->nkinds] = q;
                h->kind_mass[h->nkinds] = m;
            }
            found = h->nkinds++;
        }
        kind[i] = (uint8_t)(found < 255 ? found : 255);
    }
    rc = upload_pairf(h);
    if (rc) return rc;
    if (n) {
        GX_CUDA(h, cudaMemcpyAsync(h->host_stage, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        GX_LAUNCH(h, k_aos_to_soa, nblk(n, 256), 256, h->host_stage, b.x, b.y, b.z, un);
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        GX_CUDA(h, cudaMemcpyAsync(h->host_stage, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        GX_LAUNCH(h, k_aos_to_soa, nblk(n, 256), 256, h->host_stage, b.vx, b.vy, b.vz, un);
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        if (acc) {
            GX_CUDA(h, cudaMemcpyAsync(h->host_stage, acc, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            GX_LAUNCH(h, k_aos_to_soa, nblk(n, 256), 256, h->host_stage, b.ax, b.ay, b.az, un);
            GX_CUDA(h, cudaStreamSynchronize(h->stream));
        } else {
            GX_CUDA(h, cudaMemsetAsync(b.ax, 0, 3 * h->cap * sizeof(double), h->stream));
        }
        for (size_t i = 0; i < n; ++i) tmp[i] = charge ? charge[i] : h->p.charge[elem[i]];
        GX_CUDA(h, cudaMemcpyAsync(b.charge, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < n; ++i) tmp[i] = mass ? mass[i] : kElementMass[elem[i]];
        GX_CUDA(h, cudaMemcpyAsync(b.mass, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(b.elem, elem, n, cudaMemcpyHostToDevice, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(b.kind, kind.data(), n, cudaMemcpyHostToDevice, h->stream));
        if (entity)
            GX_CUDA(h, cudaMemcpyAsync(h->entity, entity, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        GX_LAUNCH(h, k_init_slots, nblk(n, 256), 256, b, h->pos_of_slot, un);
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    h->has_entity = entity != nullptr;
    double one = 1.0;
    GX_CUDA(h, cudaMemcpy(h->dscal, &one, sizeof one, cudaMemcpyHostToDevice));
    GX_CUDA(h, cudaGetLastError());
    return check_kinds(h);
}

int gx_get_state(gx_handle* h, double* pos, double* vel, double* acc) {
    int rc = require_state(h);
    if (rc) return rc;
    commit_lambda(h);
    StateBuf& b = h->buf[h->cur];
    uint32_t n = (uint32_t)h->n;
    double* outs[3] = {pos, vel, acc};
    double* srcs[3][3] = {{b.x, b.y, b.z}, {b.vx, b.vy, b.vz}, {b.ax, b.ay, b.az}};
    for (int k = 0; k < 3; ++k) {
        if (!outs[k] || !n) continue;
        GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, srcs[k][0], srcs[k][1], srcs[k][2], b.slot, h->host_stage, n);
        GX_CUDA(h, cudaMemcpyAsync(outs[k], h->host_stage, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    GX_CUDA(h, cudaGetLastError());
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    return take_step_errors(h);
}

int gx_set_bonds(gx_handle* h, size_t nbonds, const uint32_t* pairs) {
    int rc = require_state(h);
    if (rc) return rc;
    if (nbonds && !pairs) return GX_ERR_ARG;
    for (size_t k = 0; k < 2 * nbonds; ++k)
        if (pairs[k] >= h->n) return set_err(h, GX_ERR_ARG, "bond slot out of range");
    // earlier ticks on the stream may still read the list
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    if (nbonds > h->bonds_cap) {
        cudaFree(h->bonds);
        h->bonds = nullptr;
        GX_CUDA(h, cudaMalloc(&h->bonds, 2 * nbonds * sizeof(uint32_t)));
        h->bonds_cap = nbonds;
        invalidate_graphs(h);  // captured ticks hold the old buffer
    }
    unsigned long long cnt = nbonds;
    if (nbonds)
        GX_CUDA(h, cudaMemcpyAsync(h->bonds, pairs, 2 * nbonds * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                   h->stream));
    GX_CUDA(h, cudaMemcpyAsync(dnbonds(h), &cnt, sizeof cnt, cudaMemcpyHostToDevice, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    h->nbonds = nbonds;
    return GX_OK;
}

int gx_half_kick(gx_handle* h) {
    int rc = require_state(h);
    if (rc) return rc;
    const double* lam = h->lambda_pending ? h->dscal + 0 : nullptr;
    launch_kick(h, h->buf[h->cur], (uint32_t)h->n, 0.5 * h->p.dt, lam);
    if (h->lambda_pending) {
        double one = 1.0;
        GX_CUDA(h, cudaMemcpyAsync(h->dscal, &one, sizeof one, cudaMemcpyHostToDevice, h->stream));
        h->lambda_pending = false;
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_drift(gx_handle* h) {
    int rc = require_state(h);
    if (rc) return rc;
    commit_lambda(h);
    launch_drift(h, h->buf[h->cur], (uint32_t)h->n, h->p.dt);
    h->sorted = false;
    h->nl_fresh = false;
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_wrap(gx_handle* h) {
    int rc = require_state(h);
    if (rc) return rc;
    launch_wrap(h, h->buf[h->cur], (uint32_t)h->n);
    h->sorted = false;
    h->nl_fresh = false;
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_forces(gx_handle* h, double* potential, double* bond_energy, uint64_t* pairs) {
    int rc = require_state(h);
    if (rc) return rc;
    if ((rc = check_kinds(h))) return rc;
    if ((rc = settle_step_errors(h))) return rc;  // the pass reads and clears the error word
    if (h->n == 0) {  // systems/forces.rs:201-203
        if (potential) *potential = 0.0;
        if (bond_energy) *bond_energy = 0.0;
        if (pairs) *pairs = 0;
        return GX_OK;
    }
    if ((rc = rebuild_cells(h))) return rc;
    if ((rc = force_pass(h, true, potential, bond_energy, pairs, true))) return rc;
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_thermostat(gx_handle* h, double* kinetic, double* lambda) {
    int rc = require_state(h);
    if (rc) return rc;
    double tau = std::fmax(h->p.thermostat_tau, 1.0);  // thermostat.rs:26
    if (kinetic) *kinetic = 0.0;
    if (lambda) *lambda = 1.0;
    if (h->p.thermostat_temperature <= 0.0) return GX_OK;  // thermostat.rs:48-50
    commit_lambda(h);
    size_t rows = h->cap / 64 + kRedCap;
    double* kpart = h->red + 2 * rows;
    int nb = 0;
    launch_kinetic(h, h->buf[h->cur], (uint32_t)h->n, nullptr, kpart, nullptr, &nb);
    launch_thermostat_lambda(h, kpart, nb, h->p.thermal_constant, h->p.thermostat_temperature, tau,
                             (uint32_t)h->n, h->dscal + 0, h->dscal + 1);
    double out[2];
    GX_CUDA(h, cudaMemcpyAsync(out, h->dscal, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    h->lambda_pending = true;
    commit_lambda(h);
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    if (kinetic) *kinetic = out[1];
    if (lambda) *lambda = out[0];
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_stats(gx_handle* h, double* kinetic, double* speed_sum) {
    int rc = require_state(h);
    if (rc) return rc;
    size_t rows = h->cap / 64 + kRedCap;
    double* kpart = h->red + 2 * rows;
    double* spart = h->red + 3 * rows;
    int nb = 0;
    launch_kinetic(h, h->buf[h->cur], (uint32_t)h->n, h->lambda_pending ? h->dscal + 0 : nullptr, kpart, spart, &nb);
    launch_finalize_sum(h, kpart, nb, h->dscal + 1);
    launch_finalize_sum(h, spart, nb, h->dscal + 4);
    double out[5];
    GX_CUDA(h, cudaMemcpyAsync(out, h->dscal, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    if (kinetic) *kinetic = out[1];
    if (speed_sum) *speed_sum = out[4];
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

namespace {
// gx_step's body.  With `defer` (gx_tick_host) the ticks are only queued:
// the record stays on the device and nothing waits for the stream.
int step_impl(gx_handle* h, int nsteps, gx_tick_stats* stats, int use_graph, bool defer) {
    int rc = require_state(h);
    if (rc) return rc;
    if (nsteps < 0) return GX_ERR_ARG;
    if ((rc = check_kinds(h))) return rc;
    (void)use_graph;
    const bool fresh0 = h->nl_fresh;
    h->nl_fresh = false;  // set again below once the ticks ran on the list path
    uint32_t n = (uint32_t)h->n;
    bool thermo = h->p.enable_thermostat && h->p.thermostat_temperature > 0.0;
    double tau = std::fmax(h->p.thermostat_tau, 1.0);
    size_t rows = h->cap / 64 + kRedCap;
    double* kpart = h->red + 2 * rows;
    double* spart = h->red + 3 * rows;
    gx_tick_stats* drec = nullptr;
    if (stats && nsteps) {
        // per-tick records live in the tail of the reduction buffer
        drec = (gx_tick_stats*)(h->red + 4 * rows);
        if ((size_t)nsteps * sizeof(gx_tick_stats) > 2 * rows * sizeof(double)) {
            // record in chunks
            int done = 0;
            int chunk = (int)(2 * rows * sizeof(double) / sizeof(gx_tick_stats));
            while (done < nsteps) {
                int k = nsteps - done < chunk ? nsteps - done : chunk;
                if ((rc = gx_step(h, k, stats + done, use_graph))) return rc;
                done += k;
            }
            return GX_OK;
        }
    }
    // One tick.  With `uniform` the launch sequence does not depend on host
    // state, so it can be captured: the first kick always applies the lambda
    // slot (1.0 unless a Berendsen scale is pending; v * 1.0 == v) and resets it.
    const bool use_nl = n && (h->kernel_variant >= 5 || h->kernel_variant == 0) && nl_eligible(h);
    if (n && (rc = ensure_sort_tmp(h, h->cl, h->cap))) return rc;  // a captured re-sort must not allocate
    if (n && h->p.enable_collisions && (rc = collide_prepare(h))) return rc;  // CollisionSystem: allocate first
    if (use_nl) {
        bool stale = false;
        if ((rc = nl_prepare(h, &stale))) return rc;
        if (stale) invalidate_graphs(h);
    }
    // One tick of the neighbour-list path (gx_nlist.cu): no buffer flip.
    auto tick_nl = [&](bool uniform) -> int {
        const bool pend = uniform || h->lambda_pending;
        int nb = 0;
        // the potential and pair count only where a record takes them; the
        // record's K and speed sum come from the finish kernel's partials
        int r = nl_tick(h, pend ? h->dscal + 0 : nullptr, (thermo || drec) ? kpart : nullptr, drec ? spart : nullptr,
                        &nb, drec != nullptr);
        if (r) return r;
        // the scale slot back to 1 once applied; with the thermostat on, its
        // kernel below overwrites the slot anyway
        if (pend && !thermo) GX_LAUNCH(h, k_fill_d, 1, 32, h->dscal, 1, 1.0);
        h->lambda_pending = false;
        if (thermo) {  // on a recorded tick its sum of the partials is also the record's K
            launch_thermostat_lambda(h, kpart, nb, h->p.thermal_constant, h->p.thermostat_temperature, tau, n,
                                     h->dscal + 0, drec ? h->dscal + 1 : nullptr);
            h->lambda_pending = true;
        }
        if (drec) {  // K and the speed sum of the scaled v: lambda^2 K and lambda S of the kicked v
            if (!thermo) launch_finalize_sum(h, kpart, nb, h->dscal + 1);
            GX_LAUNCH(h, k_record_sum, 1, kRecThreads, spart, nb, drec, h->dscal, h->dcount, thermo ? 1 : 0,
                      thermo ? 1 : 0);
        }
        return GX_OK;
    };
    auto tick = [&](bool uniform) -> int {
        if (use_nl) return tick_nl(uniform);
        const bool pend = uniform || h->lambda_pending;
        // VelocityHalfKick, with the previous tick's pending thermostat scale
        launch_kick(h, h->buf[h->cur], n, 0.5 * h->p.dt, pend ? h->dscal + 0 : nullptr);
        if (pend) GX_LAUNCH(h, k_fill_d, 1, 32, h->dscal, 1, 1.0);
        h->lambda_pending = false;
        launch_drift(h, h->buf[h->cur], n, h->p.dt);                    // PositionDrift
        if (h->p.enable_boundaries) launch_wrap(h, h->buf[h->cur], n);  // BoundarySystem
        if (n) {                                                        // ForceSystem
            int r = rebuild_cells(h);
            if (!r) r = force_pass(h, true, nullptr, nullptr, nullptr, false);
            if (!r && h->p.enable_collisions) r = collide_pass(h);     // CollisionSystem
            if (r) return r;
        }
        launch_kick(h, h->buf[h->cur], n, 0.5 * h->p.dt, nullptr);  // VelocityHalfKick
        if (thermo) {                                              // ThermostatSystem
            int nb = 0;
            launch_kinetic(h, h->buf[h->cur], n, nullptr, kpart, nullptr, &nb);
            launch_thermostat_lambda(h, kpart, nb, h->p.thermal_constant, h->p.thermostat_temperature, tau, n,
                                     h->dscal + 0, nullptr);
            h->lambda_pending = true;
        }
        if (drec) {
            int nb = 0;
            launch_kinetic(h, h->buf[h->cur], n, h->lambda_pending ? h->dscal + 0 : nullptr, kpart, spart, &nb);
            launch_finalize_sum(h, kpart, nb, h->dscal + 1);
            launch_finalize_sum(h, spart, nb, h->dscal + 4);
            GX_LAUNCH(h, k_record, 1, 1, drec, h->dscal, h->dcount, thermo ? 1 : 0, 0);
        }
        return GX_OK;
    };
    if (drec) GX_CUDA(h, cudaMemsetAsync(h->dcount + 5, 0, sizeof(unsigned long long), h->stream));
    const bool graph = use_graph && n && !h->prof_on;
    const uint64_t key = ((uint64_t)n << 20) ^ ((uint64_t)h->precision << 1) ^ ((uint64_t)h->kernel_variant << 3) ^
                         ((uint64_t)bonds_on(h) << 6) ^ ((uint64_t)thermo << 7) ^ ((uint64_t)h->cap << 8) ^
                         ((uint64_t)use_nl << 62) ^ 1u;
    // kTicksPerGraph list ticks as one graph (capture only: nothing runs);
    // the host-side pending-scale flag is left as a captured run leaves it
    auto capture_multi = [&](int rs) -> int {
        if (h->graph_multi[rs]) cudaGraphExecDestroy(h->graph_multi[rs]);
        h->graph_multi[rs] = nullptr;
        const uint64_t l0 = h->launches;
        const bool pend0 = h->lambda_pending;
        GX_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int trc = GX_OK;
        for (int k = 0; k < kTicksPerGraph && !trc; ++k) trc = tick(true);
        cudaGraph_t gr = nullptr;
        cudaError_t ce = cudaStreamEndCapture(h->stream, &gr);
        if (trc || ce != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            h->lambda_pending = pend0;
            h->launches = l0;
            return trc ? trc : cuda_err(h, ce, "cudaStreamEndCapture");
        }
        cudaGraphExec_t ex = nullptr;
        ce = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        if (ce != cudaSuccess) return cuda_err(h, ce, "cudaGraphInstantiate");
        h->graph_multi[rs] = ex;
        h->graph_multi_key[rs] = key;
        h->graph_multi_kernels[rs] = h->launches - l0;
        h->launches = l0;
        return GX_OK;
    };
    for (int s = 0; s < nsteps; ++s) {
        if (!graph) {
            if ((rc = tick(false))) return rc;
            continue;
        }
        const int par = h->cur, rs = drec ? 1 : 0;
        if (use_nl && nsteps - s >= kTicksPerGraph) {  // the list path keeps one buffer: ticks chain as captured
            if (!(h->graph_multi[rs] && h->graph_multi_key[rs] == key) && (rc = capture_multi(rs))) return rc;
            GX_CUDA(h, cudaGraphLaunch(h->graph_multi[rs], h->stream));
            h->launches += h->graph_multi_kernels[rs];
            h->lambda_pending = thermo;
            s += kTicksPerGraph - 1;
            continue;
        }
        if (h->graph_exec[par][rs] && h->graph_key[par][rs] == key) {
            GX_CUDA(h, cudaGraphLaunch(h->graph_exec[par][rs], h->stream));
            h->launches += h->graph_kernels[par][rs];
            if (!use_nl) {
                h->cur ^= 1;  // the captured tick rebuilt the cell list into the other buffer
                h->sorted = true;
            }
            h->lambda_pending = thermo;
            continue;
        }
        if (!use_nl && !h->sorted) {  // first tick runs eagerly: every buffer it needs gets allocated
            if ((rc = tick(true))) return rc;
            continue;
        }
        if (h->graph_exec[par][rs]) cudaGraphExecDestroy(h->graph_exec[par][rs]);
        h->graph_exec[par][rs] = nullptr;
        const uint64_t l0 = h->launches;
        const bool pend0 = h->lambda_pending;
        GX_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int trc = tick(true);
        cudaGraph_t gr = nullptr;
        cudaError_t ce = cudaStreamEndCapture(h->stream, &gr);
        if (trc || ce != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            if (!use_nl) h->cur ^= 1;  // capture did not execute: undo the host-side effects
            h->lambda_pending = pend0;
            return trc ? trc : cuda_err(h, ce, "cudaStreamEndCapture");
        }
        cudaGraphExec_t ex = nullptr;
        ce = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        if (ce != cudaSuccess) return cuda_err(h, ce, "cudaGraphInstantiate");
        h->graph_exec[par][rs] = ex;
        h->graph_key[par][rs] = key;
        h->graph_kernels[par][rs] = h->launches - l0;
        // the list path's multi-tick graph is captured with the single one, so
        // that any call that captures (a warm-up) leaves both ready
        if (use_nl && !(h->graph_multi[rs] && h->graph_multi_key[rs] == key)) {
            const uint64_t l1 = h->launches;
            const bool pend1 = h->lambda_pending;
            h->lambda_pending = pend0;  // as before the single tick's capture
            int mrc = capture_multi(rs);
            h->lambda_pending = pend1;
            h->launches = l1;
            if (mrc) return mrc;
        }
        GX_CUDA(h, cudaGraphLaunch(ex, h->stream));  // the captured tick has not run yet: run it now
    }
    if (use_nl) h->sorted = false;  // buf[cur] is ordered by the list grid, not the force grid
    h->nl_fresh = nsteps > 0 ? (use_nl && h->nl_valid) : fresh0;
    h->last_tick_nl = use_nl;
    if (defer) return GX_OK;
    if (drec) {
        GX_CUDA(h, cudaMemcpyAsync(stats, drec, (size_t)nsteps * sizeof(gx_tick_stats), cudaMemcpyDeviceToHost,
                                   h->stream));
    }
    if (h->step_async && !drec && h->herr) {
        // no wait: the error word follows in stream order, read by the next waiting call
        GX_CUDA(h, cudaMemcpyAsync(h->herr, h->derr, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaGetLastError());
        h->step_errs_pending = true;
        return GX_OK;
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    h->step_errs_pending = false;
    uint32_t e = 0;
    GX_CUDA(h, cudaMemcpy(&e, h->derr, sizeof e, cudaMemcpyDeviceToHost));
    return step_error(h, e);
}
}  // namespace

int gx_step(gx_handle* h, int nsteps, gx_tick_stats* stats, int use_graph) {
    return step_impl(h, nsteps, stats, use_graph, false);
}

int gx_collisions(gx_handle* h, uint64_t* collisions) {
    int rc = require_state(h);
    if (rc) return rc;
    if (collisions) *collisions = 0;
    if ((rc = collide_prepare(h)) || (rc = commit_lambda(h)) || (rc = collide_pass(h))) return rc;
    unsigned long long pass = 0, total = 0;
    if ((rc = collide_read(h, &pass, &total))) return rc;
    GX_CUDA(h, cudaGetLastError());
    if (collisions) *collisions = pass;
    return GX_OK;
}

int gx_set_kernel_variant(gx_handle* h, int variant) {
    if (!h || variant < 0 || variant > 8) return GX_ERR_ARG;
    h->kernel_variant = variant;
    invalidate_graphs(h);
    return GX_OK;
}

int gx_autotune(gx_handle* h, int reps, int* best, double* ms) {
    int rc = require_state(h);
    if (rc) return rc;
    if (reps < 1) reps = 1;
    for (int v = 0; v < 9; ++v)
        if (ms) ms[v] = -1.0;
    if (h->precision != GX_MIXED || h->n == 0) {
        if (best) *best = h->kernel_variant;
        return GX_OK;
    }
    // Each variant produces the same fixed-point sums, so repeated force
    // passes leave the state bit-identical whichever variant runs.
    const int cand[4] = {4, 1, 3, 2};
    int pick = 4;
    double best_ms = 1e300;
    const int saved = h->kernel_variant;
    for (int v : cand) {
        const GridGeom& g = h->fgrid;
        if ((v == 2 || v == 3) && (g.n[0] < 3 || g.n[1] < 3 || g.n[2] < 3)) continue;
        h->kernel_variant = v;
        if ((rc = gx_forces(h, nullptr, nullptr, nullptr))) break;  // warm-up
        if ((rc = gx_timer_mark(h, 14))) break;
        for (int r = 0; r < reps && !rc; ++r) rc = force_pass(h, true, nullptr, nullptr, nullptr, false);
        if (rc || (rc = gx_timer_mark(h, 15))) break;
        double t = 0.0;
        if ((rc = gx_timer_elapsed(h, 14, 15, &t))) break;
        t /= reps;
        if (ms) ms[v] = t;
        if (t < best_ms) {
            best_ms = t;
            pick = v;
        }
    }
    // The neighbour-list paths (variants 5-7) change the whole tick, so they
    // are compared with the best single-pass variant over full ticks, each
    // run from the same snapshot of (x, v, a, pending lambda) restored
    // afterwards.  The list skin is then chosen the same way.
    if (!rc && nl_eligible(h)) {
        const uint32_t n = (uint32_t)h->n;
        double* snap = nullptr;
        if (cudaMalloc(&snap, 9 * (size_t)n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            snap = nullptr;
        }
        if (snap) {
            const bool pend0 = h->lambda_pending;
            double lam0 = 1.0;
            StateBuf& b0 = h->buf[h->cur];
            GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, b0.x, b0.y, b0.z, b0.slot, snap, n);
            GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, b0.vx, b0.vy, b0.vz, b0.slot, snap + 3 * (size_t)n, n);
            GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, b0.ax, b0.ay, b0.az, b0.slot, snap + 6 * (size_t)n, n);
            cudaMemcpyAsync(&lam0, h->dscal, sizeof lam0, cudaMemcpyDeviceToHost, h->stream);
            cudaStreamSynchronize(h->stream);
            const int ticks = reps < 20 ? 20 : reps;  // long enough to include list rebuilds
            // ms per tick of the current configuration, state restored afterwards
            auto tick_ms = [&](double* out) -> int {
                invalidate_graphs(h);
                double t = 0.0;
                int r = GX_OK;
                if (!(r = gx_step(h, 2, nullptr, 1)) && !(r = gx_timer_mark(h, 14)) &&
                    !(r = gx_step(h, ticks, nullptr, 1)) && !(r = gx_timer_mark(h, 15)) &&
                    !(r = gx_timer_elapsed(h, 14, 15, &t)))
                    *out = t / ticks;
                StateBuf& b = h->buf[h->cur];
                GX_LAUNCH(h, k_aos_to_sorted, nblk(n, 256), 256, snap, h->pos_of_slot, b.x, b.y, b.z, n);
                GX_LAUNCH(h, k_aos_to_sorted, nblk(n, 256), 256, snap + 3 * (size_t)n, h->pos_of_slot, b.vx, b.vy,
                          b.vz, n);
                GX_LAUNCH(h, k_aos_to_sorted, nblk(n, 256), 256, snap + 6 * (size_t)n, h->pos_of_slot, b.ax, b.ay,
                          b.az, n);
                cudaMemcpyAsync(h->dscal, &lam0, sizeof lam0, cudaMemcpyHostToDevice, h->stream);
                cudaStreamSynchronize(h->stream);
                h->lambda_pending = pend0;
                h->sorted = false;
                h->nl_fresh = false;  // positions restored behind the list's back
                return r;
            };
            // each list variant with its own work shape (lanes and far-end
            // block for 5 and 6, stash for 7, brick for 8) tuned on a list
            // built for it; at small sizes the shape decides more than the
            // variant does
            const int vs[5] = {pick, 5, 6, 7, 8};
            double tt[5] = {1e300, 1e300, 1e300, 1e300, 1e300};
            int shape[5][4] = {};
            for (int q = 0; q < 5 && !rc; ++q) {
                h->kernel_variant = vs[q];
                if (vs[q] >= 5) {
                    invalidate_graphs(h);
                    if (!(rc = gx_step(h, 1, nullptr, 0))) rc = nl_tune_tpp(h, reps);
                    if (!rc) nl_shape(h, &shape[q][0], &shape[q][1], &shape[q][2], &shape[q][3]);
                }
                int r2 = tick_ms(&tt[q]);  // restores the snapshot, the tuning tick's too
                if (!rc) rc = r2;
            }
            if (ms) {
                ms[0] = tt[0] < 1e300 ? tt[0] : -1.0;
                ms[5] = tt[1] < 1e300 ? tt[1] : -1.0;
                ms[6] = tt[2] < 1e300 ? tt[2] : -1.0;
                ms[7] = tt[3] < 1e300 ? tt[3] : -1.0;
                ms[8] = tt[4] < 1e300 ? tt[4] : -1.0;
            }
            int qpick = 0;
            if (!rc) {
                for (int k = 1; k < 5; ++k)
                    if (tt[k] < tt[qpick]) qpick = k;
                pick = vs[qpick];
            }
            if (!rc && pick >= 5) {
                h->kernel_variant = pick;
                nl_set_tpp(h, shape[qpick][0]);
                nl_set_block(h, shape[qpick][1]);
                nl_set_slots(h, shape[qpick][2]);
                nl_set_brick(h, shape[qpick][3]);
                // the skin: 0.05, 0.1, 0.15 and 0.2 r_c (cell size r_c + skin)
                // over whole ticks, rebuilds included
                double skin0 = 0.0;
                nl_config(h, &skin0, nullptr);
                double best_t = 1e300, best_skin = skin0;
                const double fr[4] = {0.05, 0.1, 0.15, 0.2};
                for (int k = 0; k < 4 && !rc; ++k) {
                    const double sk = fr[k] * h->fs.rc;
                    nl_set_skin(h, sk);
                    double t = 1e300;
                    if ((rc = tick_ms(&t))) break;
                    if (t < best_t) {
                        best_t = t;
                        best_skin = sk;
                    }
                }
                nl_set_skin(h, rc ? skin0 : best_skin);
                invalidate_graphs(h);
                // threads per atom (stash size for 7, brick length for 8) of the list pass, on a list of the chosen skin
                if (!rc && !(rc = gx_step(h, 1, nullptr, 0))) {
                    rc = nl_tune_tpp(h, reps);
                    int r2 = tick_ms(&best_t);  // restores the snapshot after the tick above
                    if (!rc) rc = r2;
                }
            }
            cudaFree(snap);
        }
    }
    h->kernel_variant = rc ? saved : pick;
    invalidate_graphs(h);
    if (best) *best = h->kernel_variant;
    return rc;
}

int gx_set_list_skin(gx_handle* h, double skin) {
    if (!h || !(skin >= 0.0) || !std::isfinite(skin)) return GX_ERR_ARG;
    invalidate_graphs(h);
    return nl_set_skin(h, skin);
}

}  // extern "C"

namespace gx {
// The device bond list and its device count were rewritten in place (bond
// observation): captured ticks stay valid unless the buffer changed.
void bonds_changed(gx_handle* h, size_t nbonds, bool realloc) {
    if (realloc) invalidate_graphs(h);
    h->nbonds = nbonds;
}
}  // namespace gx

extern "C" {

int gx_get_list_config(gx_handle* h, double* skin, int* threads_per_atom) {
    if (!h) return GX_ERR_ARG;
    return nl_config(h, skin, threads_per_atom);
}

int gx_set_list_threads(gx_handle* h, int threads_per_atom) {
    if (!h) return GX_ERR_ARG;
    invalidate_graphs(h);
    return nl_set_tpp(h, threads_per_atom);
}

int gx_set_list_stash(gx_handle* h, int slots) {
    if (!h) return GX_ERR_ARG;
    invalidate_graphs(h);
    return nl_set_slots(h, slots);
}

int gx_set_list_block(gx_handle* h, int threads) {
    if (!h) return GX_ERR_ARG;
    invalidate_graphs(h);
    return nl_set_block(h, threads);
}

int gx_get_list_shape(gx_handle* h, int* threads_per_atom, int* block, int* stash_slots, int* brick_cells) {
    if (!h || !threads_per_atom || !block || !stash_slots || !brick_cells) return GX_ERR_ARG;
    return nl_shape(h, threads_per_atom, block, stash_slots, brick_cells);
}

int gx_set_list_brick(gx_handle* h, int cells) {
    if (!h) return GX_ERR_ARG;
    invalidate_graphs(h);
    return nl_set_brick(h, cells);
}

int gx_list_stats(gx_handle* h, uint64_t* entries, uint64_t* overflowed_atoms) {
    if (!h || !entries || !overflowed_atoms) return GX_ERR_ARG;
    return nl_stats(h, entries, overflowed_atoms);
}

int gx_set_pass_timing(gx_handle* h, int on) {
    if (!h) return GX_ERR_ARG;
    if (on && !h->pass_ev[0]) {
        GX_CUDA(h, cudaEventCreate(&h->pass_ev[0]));
        GX_CUDA(h, cudaEventCreate(&h->pass_ev[1]));
    }
    h->pass_timing = on != 0;
    invalidate_graphs(h);  // the captured ticks gain or lose the event nodes
    return GX_OK;
}

int gx_pass_ms(gx_handle* h, double* ms) {
    if (!h || !ms) return GX_ERR_ARG;
    if (!h->pass_ev[0]) return set_err(h, GX_ERR_STATE, "pass timing was never switched on");
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    float t = 0.f;
    GX_CUDA(h, cudaEventElapsedTime(&t, h->pass_ev[0], h->pass_ev[1]));
    *ms = t;
    return GX_OK;
}

int gx_list_rebuilds(gx_handle* h, uint64_t* rebuilds) {
    if (!h || !rebuilds) return GX_ERR_ARG;
    return nl_rebuilds(h, rebuilds);
}

int gx_set_dynamic(gx_handle* h, const double* pos, const double* vel, const double* acc) {
    int rc = require_state(h);
    if (rc) return rc;
    if (h->lambda_pending) {  // the host columns replace v: the pending scale is void
        GX_LAUNCH(h, k_fill_d, 1, 32, h->dscal, 1, 1.0);
        h->lambda_pending = false;
    }
    StateBuf& b = h->buf[h->cur];
    uint32_t n = (uint32_t)h->n;
    const double* ins[3] = {pos, vel, acc};
    double* dsts[3][3] = {{b.x, b.y, b.z}, {b.vx, b.vy, b.vz}, {b.ax, b.ay, b.az}};
    for (int k = 0; k < 3; ++k) {
        if (!ins[k] || !n) continue;
        double* stage = h->host_stage;
        GX_CUDA(h, cudaMemcpyAsync(stage, ins[k], 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        GX_LAUNCH(h, k_aos_to_sorted, nblk(n, 256), 256, stage, h->pos_of_slot, dsts[k][0], dsts[k][1], dsts[k][2], n);
    }
    if (pos) {
        h->sorted = false;
        h->nl_fresh = false;
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

// One tick against host columns: gx_set_dynamic, gx_step(h, 1, stats, 1)
// and gx_get_state in one call, with the same results, and with the copies
// overlapped.  The columns cross PCIe on a stream of their own: each one is
// scattered to the sorted order as soon as it lands, and on the list path
// the positions go back while the pair pass runs (a list tick records
// io_ev[3] once they are final); velocities and accelerations follow the
// tick.
int gx_tick_host(gx_handle* h, double* pos, double* vel, double* acc, gx_tick_stats* stats) {
    int rc = require_state(h);
    if (rc) return rc;
    if (!pos || !vel || !acc) return set_err(h, GX_ERR_ARG, "gx_tick_host needs the position, velocity and "
                                                            "acceleration columns");
    if ((rc = settle_step_errors(h))) return rc;
    if (!h->io_stream) {
        GX_CUDA(h, cudaStreamCreateWithFlags(&h->io_stream, cudaStreamNonBlocking));
        for (cudaEvent_t& e : h->io_ev) GX_CUDA(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (!h->io_events) {
        h->io_events = true;
        invalidate_graphs(h);  // the captured list ticks gain the positions-final event
    }
    if (h->io_cap < h->cap) {
        GX_CUDA(h, cudaStreamSynchronize(h->io_stream));
        cudaFree(h->io_stage);
        h->io_stage = nullptr;
        h->io_cap = 0;
        GX_CUDA(h, cudaMalloc(&h->io_stage, 9 * h->cap * sizeof(double)));
        h->io_cap = h->cap;
    }
    const uint32_t n = (uint32_t)h->n;
    const size_t bytes = 3 * (size_t)n * sizeof(double);
    double* st[3] = {h->io_stage, h->io_stage + 3 * h->io_cap, h->io_stage + 6 * h->io_cap};
    cudaStream_t ms = h->stream, io = h->io_stream;
    // From the first queued copy on, a failure waits for both streams before
    // it returns, so that no queued work still reads the caller's columns.
    auto fail = [&](int r) -> int {
        h->stream = ms;
        cudaStreamSynchronize(io);
        cudaStreamSynchronize(ms);
        return r;
    };
#define GX_IO(call)                                                  \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return fail(cuda_err(h, e_, #call));  \
    } while (0)
    if (h->lambda_pending) {  // the host columns replace v: the pending scale is void
        GX_LAUNCH(h, k_fill_d, 1, 32, h->dscal, 1, 1.0);
        h->lambda_pending = false;
    }
    {
        StateBuf& b = h->buf[h->cur];
        const double* ins[3] = {pos, vel, acc};
        double* dsts[3][3] = {{b.x, b.y, b.z}, {b.vx, b.vy, b.vz}, {b.ax, b.ay, b.az}};
        for (int k = 0; k < 3; ++k) {
            if (!n) break;
            GX_IO(cudaMemcpyAsync(st[k], ins[k], bytes, cudaMemcpyHostToDevice, io));
            GX_IO(cudaEventRecord(h->io_ev[k], io));
            GX_IO(cudaStreamWaitEvent(ms, h->io_ev[k], 0));
            GX_LAUNCH(h, k_aos_to_sorted, nblk(n, 256), 256, st[k], h->pos_of_slot, dsts[k][0], dsts[k][1],
                      dsts[k][2], n);
        }
        h->sorted = false;
        h->nl_fresh = false;
    }
    if ((rc = step_impl(h, 1, stats, 1, true))) return fail(rc);
    if (n) {
        StateBuf& b = h->buf[h->cur];
        if (h->last_tick_nl) {  // positions final at io_ev[3]: gathered and copied beside the pair pass
            GX_IO(cudaStreamWaitEvent(io, h->io_ev[3], 0));
            h->stream = io;
            GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, b.x, b.y, b.z, b.slot, st[0], n);
            h->stream = ms;
        } else {
            GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, b.x, b.y, b.z, b.slot, st[0], n);
            GX_IO(cudaEventRecord(h->io_ev[0], ms));
            GX_IO(cudaStreamWaitEvent(io, h->io_ev[0], 0));
        }
        GX_IO(cudaGetLastError());
        GX_IO(cudaMemcpyAsync(pos, st[0], bytes, cudaMemcpyDeviceToHost, io));
        if ((rc = commit_lambda(h))) return fail(rc);
        double* srcs[2][3] = {{b.vx, b.vy, b.vz}, {b.ax, b.ay, b.az}};
        double* outs[2] = {vel, acc};
        for (int k = 0; k < 2; ++k) {
            GX_LAUNCH(h, k_soa_to_aos, nblk(n, 256), 256, srcs[k][0], srcs[k][1], srcs[k][2], b.slot, st[k + 1], n);
            GX_IO(cudaEventRecord(h->io_ev[k + 1], ms));
            GX_IO(cudaStreamWaitEvent(io, h->io_ev[k + 1], 0));
            GX_IO(cudaMemcpyAsync(outs[k], st[k + 1], bytes, cudaMemcpyDeviceToHost, io));
        }
    }
    GX_IO(cudaGetLastError());
    GX_IO(cudaStreamSynchronize(io));
    GX_IO(cudaStreamSynchronize(ms));
    if (stats) {
        size_t rows = h->cap / 64 + kRedCap;
        GX_IO(cudaMemcpy(stats, h->red + 4 * rows, sizeof(gx_tick_stats), cudaMemcpyDeviceToHost));
    }
#undef GX_IO
    h->step_errs_pending = false;
    uint32_t e = 0;
    GX_CUDA(h, cudaMemcpy(&e, h->derr, sizeof e, cudaMemcpyDeviceToHost));
    return step_error(h, e);
}

int gx_synchronize(gx_handle* h) {
    if (!h) return GX_ERR_ARG;
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    return take_step_errors(h);
}

int gx_set_step_async(gx_handle* h, int on) {
    if (!h) return GX_ERR_ARG;
    if (on && !h->herr) GX_CUDA(h, cudaMallocHost(&h->herr, sizeof(uint32_t)));
    if (!on) {  // report what an earlier step left before going back to waiting steps
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        int rc = take_step_errors(h);
        h->step_async = false;
        return rc;
    }
    h->step_async = true;
    return GX_OK;
}

int gx_timer_mark(gx_handle* h, int slot) {
    if (!h || slot < 0 || slot >= 16) return GX_ERR_ARG;
    if (!h->timers[slot]) GX_CUDA(h, cudaEventCreate(&h->timers[slot]));
    GX_CUDA(h, cudaEventRecord(h->timers[slot], h->stream));
    return GX_OK;
}

int gx_timer_elapsed(gx_handle* h, int a, int b, double* ms) {
    if (!h || !ms || a < 0 || b < 0 || a >= 16 || b >= 16 || !h->timers[a] || !h->timers[b]) return GX_ERR_ARG;
    GX_CUDA(h, cudaEventSynchronize(h->timers[b]));
    float t = 0.f;
    GX_CUDA(h, cudaEventElapsedTime(&t, h->timers[a], h->timers[b]));
    *ms = (double)t;
    return GX_OK;
}

uint64_t gx_launch_count(const gx_handle* h) { return h ? h->launches : 0; }

int gx_measure_fp32_peak(int device, double* tflops) {
    if (!tflops) return GX_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GX_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float* out = nullptr;
    if (cudaMalloc(&out, 1024 * 1024 * sizeof(float)) != cudaSuccess) return GX_ERR_OOM;
    const int iters = 4096, threads = 512, blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_fma_peak<<<blocks, threads>>>(out, iters, 1.0f);  // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a);
        k_fma_peak<<<blocks, threads>>>(out, iters, 1.0f + rep * 1e-7f);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        // 8 independent FMA chains x iters per thread, 2 FLOP per FMA
        double flop = 2.0 * 8.0 * iters * (double)threads * blocks;
        double tf = flop / (t * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaError_t e = cudaGetLastError();
    cudaFree(out);
    if (e != cudaSuccess) return GX_ERR_CUDA;
    *tflops = best;
    return GX_OK;
}

int gx_measure_fp64_peak(int device, double* tflops) {
    if (!tflops) return GX_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GX_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double* out = nullptr;
    if (cudaMalloc(&out, 1024 * sizeof(double)) != cudaSuccess) return GX_ERR_OOM;
    const int iters = 2048, threads = 512, blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_fma_peak_f64<<<blocks, threads>>>(out, iters, 1.0);  // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(a);
        k_fma_peak_f64<<<blocks, threads>>>(out, iters, 1.0 + rep * 1e-9);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        double flop = 2.0 * 8.0 * iters * (double)threads * blocks;  // 8 FMA chains, 2 FLOP per FMA
        double tf = flop / (t * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaError_t e = cudaGetLastError();
    cudaFree(out);
    if (e != cudaSuccess) return GX_ERR_CUDA;
    *tflops = best;
    return GX_OK;
}

int gx_profile_enable(gx_handle* h, int on) {
    if (!h) return GX_ERR_ARG;
    h->prof_on = on != 0;
    return GX_OK;
}

int gx_profile_read(gx_handle* h, const char** names, uint64_t* launches, double* ms, int cap, int reset) {
    if (!h) return GX_ERR_ARG;
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    int k = 0;
    for (auto& s : h->prof) {
        for (size_t q = 0; q + 1 < s.ev.size(); q += 2) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, s.ev[q], s.ev[q + 1]) == cudaSuccess) s.ms += t;
            h->ev_pool.push_back(s.ev[q]);
            h->ev_pool.push_back(s.ev[q + 1]);
        }
        s.ev.clear();
        if (k < cap) {
            if (names) names[k] = s.name;
            if (launches) launches[k] = s.launches;
            if (ms) ms[k] = s.ms;
        }
        ++k;
        if (reset) {
            s.launches = 0;
            s.ms = 0.0;
        }
    }
    return k;
}

}  // extern "C"
