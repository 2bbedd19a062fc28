// mmff_world.cu -- device-resident world of many MMFF systems and the C-ABI
// that drives it (declared in include/MMFFmulti_lib.h).
//
// The host side packs systems of uneven size back to back (CSR offsets), moves
// each system into a local frame (positions relative to its own centroid, so
// FP32 coordinates keep ~5e-7 A resolution), converts the force-field
// parameters to the FP32 layout the kernels read, groups systems into size
// buckets and launches one persistent relaxation kernel per bucket.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "MMFFmulti_lib.h"
#include "mmff_device.cuh"
#include "mmff_host.h"
#include "mmff_world.h"

namespace mmff {
// kernels (mmff_relax.cu, mmff_grid.cu)
template <int T, int S, bool C> __global__ void relax_kernel(Params, Systems, const int*, int, int*, int, int);
template <int T, int S, bool E> __global__ void eval_kernel(Params, Systems, const int*, int, int, int);
__global__ void grid_sample_kernel(Params, int, const float4*, const float4*, float4*);
__global__ void grid_potential_kernel(int, int, int, double3, double3, int, const double4*, const double2*,
                                      const double3*, int, const double3*, int, double, double*);
__global__ void solve_open_kernel(double*, long, int, long, long, int, long, double*);
__global__ void solve_periodic_kernel(double*, long, int, long, long, int, long, double*);
__global__ void pack_grid_kernel(long, const double*, float4*);
void* relax_fn(int T, int S, bool count);
void* eval_fn(int T, int S, bool energy);
void* relax_warp_fn(int apl, bool count);
void* relax_explore_fn(int T);
void* relax_warp_explore_fn(int apl);
void* eval_warp_fn(int apl, bool energy);

}  // namespace mmff

using namespace mmff;

namespace {

std::string g_err;
// kernels this library launched (relaxation, evaluation, learned proposal);
// a graph replay counts every kernel node it runs
std::atomic<unsigned long long> g_launches{0};
bool g_capturing = false;      // enqueue_relax inside a graph capture: counted at replay
int fail(const char* fmt, ...) {
    char buf[512];
    va_list ap; va_start(ap, fmt); vsnprintf(buf, sizeof buf, fmt, ap); va_end(ap);
    g_err = buf;
    return -1;
}
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail("%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, __LINE__); } while (0)

template <class X> struct DBuf {
    X* p = nullptr; size_t n = 0;
    int ensure(size_t cnt) {
        if (cnt <= n && p) return 0;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        if (cnt == 0) return 0;
        cudaError_t e = cudaMalloc(&p, cnt * sizeof(X));
        if (e != cudaSuccess) return fail("cudaMalloc(%zu B): %s", cnt * sizeof(X), cudaGetErrorString(e));
        n = cnt;
        return 0;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

struct Bucket {
    int kind = 0;                  // 0: CTA per system (T threads, S lanes per atom); 1: warp per system
    int apl = 1;                   // warp engine: atoms per lane (1: <=32 atoms, 2: <=64)
    int T = 64, S = 1, maxNA = 0, maxNN = 0;
    std::vector<int> sys;          // system indices, largest first
    DBuf<int> queue;
    int smem = 0, grid = 0;
    int cls = 0;                   // size class (see size_class)
    // CTA relax kernels with a cutoff and a 2-D cell: scratch for the shifted-image
    // pair lists, vstride 32-bit words per resident CTA (0: none)
    DBuf<uint32_t> vl;
    int vstride = 0;
};

// autotuned launch configuration of one size class (kind -1: heuristic)
struct Tune {
    int kind = -1, apl = 1, T = 0, S = 0;
    float us_per_sys_step = 0.f;
};

struct World {
    bool ready = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> bstreams;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evfork = nullptr;
    std::vector<cudaEvent_t> bev;
    // grid
    DBuf<float4> grid;
    int gn[3] = {0, 0, 0};
    double gpos0[3] = {0, 0, 0}, gstep[3] = {1, 1, 1};
    // systems
    int nsys = 0, NA = 0, NN = 0, NV = 0;
    std::vector<int> natoms, nnode;
    std::vector<int4> desc;
    std::vector<double> orig;      // [nsys*3]
    DBuf<int4> d_desc; DBuf<int> d_nnode; DBuf<float> d_lvec; DBuf<float4> d_gorg;
    DBuf<float4> d_REQ, d_PLQ; DBuf<int4> d_ng, d_ngC, d_bk;
    DBuf<float4> d_apar, d_bL, d_bK, d_ksp, d_kpp;
    // 1-3 pairs and central-image exclusion rows (built for the current flags and image set)
    std::vector<int4> h_ng, h_ngC;
    std::vector<int> h_a13;
    DBuf<int> d_a13, d_moff;
    DBuf<uint32_t> d_xmask;
    // position springs (relax only)
    DBuf<float4> d_constr, d_constrK;
    bool has_constr = false;
    bool pair_lists = true;        // shifted-image pair lists in the CTA relax kernels (mmff_set_pair_lists)
    double list_skin = 1.0;        // their skin [A]
    // distance / angle constraints (mmff_set_bond_constraints)
    DBuf<int4> d_dci, d_aci;
    DBuf<float4> d_dca, d_dcb, d_aca;
    int ndcon = 0, nacon = 0;
    // per-atom GridFF stencil cache of the CTA engine (grid_slice_cached)
    DBuf<unsigned int> d_gkey; DBuf<float4> d_gcs;
    bool gcache = true;            // mmff_set_grid_cache
    DBuf<float4> d_pos, d_vel, d_force, d_pos0, d_vel0;
    DBuf<double4> d_fire, d_fire0, d_energy;
    DBuf<int> d_status, d_nsteps, d_counter;
    DBuf<unsigned long long> d_stats;
    bool count = false;
    DBuf<float> d_fconv;
    // parameters
    int flags = F_BONDS | F_PIPI | F_PISIGMA | F_ANGLES | F_SUB_ANGLE_NB | F_NONBONDED | F_GRID | F_PBC;
    int npbc[3] = {1, 1, 0};
    double Rcut = -1.0, alphaMorse = 1.5, FmaxNB = 10.0;
    double fire[10] = {0.1, 0.01, 0.1, 1.1, 0.5, 0.8, 3, 0.0, -1.0, 0};  // dt_max dt_min damp_max finc fdec falpha minLastNeg cv_kill Flim variant
    // launch configuration (0 = heuristic)
    int force_T = 0, force_S = 0;
    std::vector<Bucket> buckets;
    bool buckets_dirty = true;
    Tune tune[6];
    // relax graph
    bool use_graph = false, graph_valid = false;
    cudaGraphExec_t gexec = nullptr;
    int gkey_nstep = 0, gkey_mode = 0, gkey_version = -1;
    bool gkey_count = false;
    double gkey_fconv = 0.0;
    int version = 0;               // bumped by every change of parameters or systems
    // direct substrate term
    DBuf<float4> d_spos, d_sREQ;
    int nsurf = 0, snpbc[3] = {1, 1, 0};
    float slv[9] = {0};
    double sRdamp = 1.0;
    // Langevin drive
    double md_dt = 0.05, md_gamma = 0.1, md_T = 300.0;
    unsigned long long md_seed = 12345;
    int md_step = 0;
    // exploring cycle (mmff_set_explore; n_explore < 0: not set up for the current systems)
    DBuf<int4> d_gopt;
    DBuf<float4> d_minpos;
    int n_explore = -1, n_relax = 0;
};

World W;

int ensure_ready() {
    if (W.ready) return 0;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail("no CUDA device available (%s)", cudaGetErrorString(e));
    CK(cudaSetDevice(W.device));
    CK(cudaStreamCreateWithFlags(&W.stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&W.ev0));
    CK(cudaEventCreate(&W.ev1));
    CK(cudaEventCreateWithFlags(&W.evfork, cudaEventDisableTiming));
    W.ready = true;
    return 0;
}

Params make_params(bool for_eval, int nstep_max, double Fconv, int conv_mode) {
    Params P;
    memset(&P, 0, sizeof P);
    P.flags = W.flags & ~F_EXCL13;
    if (excl13_active(P.flags)) P.flags |= F_EXCL13;
    P.flags &= ~F_CONSTR;
    if (W.has_constr && !for_eval) P.flags |= F_CONSTR;
    P.flags &= ~F_BCONS;
    if ((W.ndcon || W.nacon) && !for_eval) P.flags |= F_BCONS;
    if (!W.grid.p) P.flags &= ~F_GRID;
    for (int k = 0; k < 3; k++) P.npbc[k] = W.npbc[k];
    P.Rc2 = W.Rcut > 0 ? (float)(W.Rcut * W.Rcut) : 0.f;
    P.kq_rc2 = W.Rcut > 0 ? (float)(1.0 / (W.Rcut * W.Rcut)) : 0.f;
    P.Fmax2NB = (float)(W.FmaxNB * W.FmaxNB);
    for (int k = 0; k < 3; k++) {
        P.gn[k] = W.gn[k];
        P.ginv[k] = (float)(1.0 / W.gstep[k]);
        P.gmi[k] = (float)(-1.0 / W.gstep[k]);
    }
    P.grid = W.grid.p;
    P.dt_max = W.fire[0]; P.dt_min = W.fire[1]; P.damp_max = W.fire[2]; P.finc = W.fire[3];
    P.fdec = W.fire[4]; P.falpha = W.fire[5]; P.minLastNeg = (int)W.fire[6]; P.cv_kill = W.fire[7];
    P.Flim = for_eval ? -1.f : (float)W.fire[8];
    P.fire_variant = (int)W.fire[9];
    P.Fconv2 = Fconv * Fconv;
    P.conv_mode = conv_mode;
    P.nstep_max = nstep_max;
    if (W.nsurf > 0) {
        P.surf_pos = W.d_spos.p; P.surf_REQ = W.d_sREQ.p; P.nsurf = W.nsurf;
        for (int k = 0; k < 3; k++) { P.snpbc[k] = W.snpbc[k]; P.sg0[k] = (float)W.gpos0[k]; }
        for (int k = 0; k < 9; k++) P.slv[k] = W.slv[k];
        P.sK = (float)(-W.alphaMorse);
        P.sR2damp = (float)(W.sRdamp * W.sRdamp);
    } else {
        P.flags &= ~F_SURF;
    }
    return P;
}

Systems make_systems() {
    Systems Y;
    Y.nsys = W.nsys;
    Y.desc = W.d_desc.p; Y.nnode = W.d_nnode.p; Y.lvec = W.d_lvec.p; Y.gorg = W.d_gorg.p;
    Y.REQ = W.d_REQ.p; Y.PLQ = W.d_PLQ.p; Y.neighs = W.d_ng.p; Y.neighCell = W.d_ngC.p; Y.bkneighs = W.d_bk.p;
    Y.apars = W.d_apar.p; Y.bLs = W.d_bL.p; Y.bKs = W.d_bK.p; Y.Ksp = W.d_ksp.p; Y.Kpp = W.d_kpp.p;
    Y.a13 = W.d_a13.p; Y.xmask = W.d_xmask.p; Y.moff = W.d_moff.p;
    Y.constr = W.d_constr.p; Y.constrK = W.d_constrK.p;
    Y.dcon_i = W.d_dci.p; Y.dcon_a = W.d_dca.p; Y.dcon_b = W.d_dcb.p; Y.ndcon = W.ndcon;
    Y.acon_i = W.d_aci.p; Y.acon_a = W.d_aca.p; Y.nacon = W.nacon;
    // the cache keys pack the stencil cell into 12 + 12 + 8 bits
    const bool gc = W.gcache && W.d_gkey.p && W.gn[0] <= 4096 && W.gn[1] <= 4096 && W.gn[2] <= 256;
    Y.gkey = gc ? W.d_gkey.p : nullptr; Y.gcs = gc ? W.d_gcs.p : nullptr;
    Y.pos = W.d_pos.p; Y.vel = W.d_vel.p; Y.force = W.d_force.p; Y.fire = W.d_fire.p;
    Y.status = W.d_status.p; Y.nsteps = W.d_nsteps.p; Y.fconv = W.d_fconv.p; Y.energy = W.d_energy.p;
    Y.counters = W.d_stats.p;
    Y.gopt = W.d_gopt.p; Y.minpos = W.d_minpos.p;
    return Y;
}

int pow2_floor(int x) { int p = 1; while (p * 2 <= x) p *= 2; return p; }

// size buckets: thread count T >= atoms (<= 512); S lanes per atom in the pair sum
// size class of a system: 0/1 warp engine (<=32 / <=64 atoms), 2..5 CTA
// engine by thread count (<=64, <=128, <=256, larger)
const int kClassT[4] = {64, 128, 256, 512};
int size_class(int na) {
    if (!W.force_T && na <= 32) return 0;
    if (!W.force_T && na <= 64) return 1;
    if (W.force_T) { for (int k = 0; k < 4; k++) if (kClassT[k] == W.force_T) return 2 + k; }
    for (int k = 0; k < 4; k++) if (na <= kClassT[k]) return 2 + k;
    return 5;
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes`.  The limit
// is per function, and several buckets (or autotuner candidates) can share one
// kernel instantiation, so it only ever grows.
int set_smem_limit(void* fn, int bytes) {
    struct Seen { void* fn; int device; int bytes; };
    static std::vector<Seen> seen;
    for (auto& e : seen) {
        if (e.fn != fn || e.device != W.device) continue;
        if (bytes <= e.bytes) return 0;
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        e.bytes = bytes;
        return 0;
    }
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    seen.push_back({fn, W.device, bytes});
    return 0;
}

// launch configuration of a bucket whose systems are set: kind 1 = warp
// engine (apl atoms per lane), kind 0 = CTA engine with T threads and S lanes
// per atom in the pair sum.  Fills smem, grid; sets kernel attributes.
int config_bucket(Bucket& B, int kind, int apl, int T, int S) {
    int dev_smem = 0, nsm = 0;
    CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, W.device));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, W.device));
    B.maxNA = 0; B.maxNN = 0;
    for (int s : B.sys) { B.maxNA = std::max(B.maxNA, W.natoms[s]); B.maxNN = std::max(B.maxNN, W.nnode[s]); }
    void* fns[2];
    if (kind == 1) {
        if (B.maxNA > 32 * apl) return fail("warp engine with %d atoms per lane cannot hold %d atoms", apl, B.maxNA);
        B.kind = 1; B.apl = apl; B.T = 128; B.S = 1;
        B.smem = 4 * warp_layout(B.maxNA, B.maxNN).per_warp;
        fns[0] = relax_warp_fn(B.apl, false); fns[1] = relax_warp_fn(B.apl, true);
    } else {
        B.kind = 0; B.T = T; B.S = S;
        B.smem = smem_layout(B.maxNA, B.maxNN, B.T, W.Rcut > 0 ? shifted_images(W.flags, W.npbc) : 0).total;
        fns[0] = relax_fn(B.T, B.S, false); fns[1] = relax_fn(B.T, B.S, true);
    }
    if (B.smem > dev_smem) return fail("system too large for shared memory: %d B > %d B", B.smem, dev_smem);
    if (!fns[0] || !fns[1]) return fail("no kernel for bucket (kind %d, T=%d, S=%d)", B.kind, B.T, B.S);
    for (int f = 0; f < 2; f++) if (set_smem_limit(fns[f], B.smem)) return -1;
    void* xf = B.kind ? relax_warp_explore_fn(B.apl) : relax_explore_fn(B.T);     // exploring cycle
    if (!xf) return fail("no exploring-cycle kernel for bucket (kind %d, T=%d)", B.kind, B.T);
    if (set_smem_limit(xf, B.smem)) return -1;
    for (int e = 0; e < 2; e++) {
        void* ef = B.kind ? eval_warp_fn(B.apl, e) : eval_fn(B.T, B.S, e);
        if (set_smem_limit(ef, B.smem)) return -1;
    }
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fns[0], B.T, B.smem));
    if (occ < 1) return fail("kernel cannot be resident (T=%d smem=%d)", B.T, B.smem);
    const int per_block = B.kind ? 4 : 1;
    const int nblk = ((int)B.sys.size() + per_block - 1) / per_block;
    B.grid = std::min(nblk, occ * nsm);
    B.vstride = 0;
    if (kind == 0 && W.Rcut > 0 && B.maxNA <= 4096) {
        const int nimg = shifted_images(W.flags, W.npbc);
        if (nimg > 0 && nimg <= kListMaxImages) {
            B.vstride = B.maxNA * (kListEntriesPerAtom + 4);
            if (B.vl.ensure((size_t)B.grid * B.vstride)) return -1;
        }
    }
    if (B.queue.ensure(B.sys.size())) return -1;
    CK(cudaMemcpy(B.queue.p, B.sys.data(), B.sys.size() * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
}

// heuristic configuration of a size class: warp engine for <= 64 atoms, else
// the class's thread count with pair lanes filling the block
void default_config(int cls, int maxNA, int& kind, int& apl, int& T, int& S) {
    if (cls <= 1) { kind = 1; apl = cls + 1; T = 128; S = 1; return; }
    kind = 0; apl = 1; T = kClassT[cls - 2];
    S = std::min(pow2_floor(std::max(1, T / std::max(1, maxNA))), 8);
    if (W.force_S) S = W.force_S;
}

template <class X> int upload(DBuf<X>& d, const std::vector<X>& h) {
    if (d.ensure(h.size())) return -1;
    if (!h.empty()) CK(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(X), cudaMemcpyHostToDevice, W.stream));
    return 0;
}

// Empty every atom's GridFF stencil cache (new systems, new grid).
int clear_grid_cache() {
    if (W.d_gkey.p && W.NA > 0) CK(cudaMemsetAsync(W.d_gkey.p, 0xff, (size_t)W.NA * sizeof(unsigned int), W.stream));
    return 0;
}

// Angle pairs whose 1-3 pair the pair sum may skip (per node, bit
// angle_slot(i, j) of neighbour slots i < j): the two ends are different
// atoms, not bonded to each other, and no other angle of the system has the
// same two ends (rings of three or four atoms keep the reference's add-then-
// subtract form).  Topology only; whether the pair is central is decided per
// step from the neighbour cells.
void angle_pairs13(int na, int nn, const int4* ng, int* a13) {
    std::vector<long long> ends, bonds;
    auto key = [](int a, int b) { return a < b ? (long long)a << 32 | (unsigned)b : (long long)b << 32 | (unsigned)a; };
    for (int i = 0; i < na; i++) {
        const int g[4] = {ng[i].x, ng[i].y, ng[i].z, ng[i].w};
        for (int k = 0; k < 4; k++) if (g[k] >= 0) bonds.push_back(key(i, g[k]));
    }
    for (int ia = 0; ia < nn; ia++) {
        const int g[4] = {ng[ia].x, ng[ia].y, ng[ia].z, ng[ia].w};
        for (int i = 0; i < 3; i++) for (int j = i + 1; j < 4; j++)
            if (g[i] >= 0 && g[j] >= 0) ends.push_back(key(g[i], g[j]));
    }
    std::sort(ends.begin(), ends.end());
    std::sort(bonds.begin(), bonds.end());
    for (int ia = 0; ia < nn; ia++) {
        const int g[4] = {ng[ia].x, ng[ia].y, ng[ia].z, ng[ia].w};
        int m = 0;
        for (int i = 0; i < 3; i++) for (int j = i + 1; j < 4; j++) {
            if (g[i] < 0 || g[j] < 0 || g[i] == g[j]) continue;
            const long long k = key(g[i], g[j]);
            const auto r = std::equal_range(ends.begin(), ends.end(), k);
            if (r.second - r.first != 1 || std::binary_search(bonds.begin(), bonds.end(), k)) continue;
            m |= 1 << angle_slot(i, j);
        }
        a13[ia] = m;
    }
}

// Central-image exclusion rows of every system for the current flags and
// image set: per atom i, ceil(natoms/32) words whose bit j marks a pair the
// central-image pair sum skips -- i itself, padding slots j >= natoms, bonded
// neighbours in the central cell (NBFF.h:590-607; both directions), and with
// F_EXCL13 the central 1-3 pairs of angle_pairs13 (their angle terms carry
// them, pair13).  Rows are symmetric.
int build_xmask() {
    const bool pbc = (W.flags & F_PBC) != 0;
    const bool x13 = excl13_active(W.flags);
    const int nxi = 2 * W.npbc[0] + 1, nyi = 2 * W.npbc[1] + 1;
    const int central = (W.npbc[2] * nyi + W.npbc[1]) * nxi + W.npbc[0];
    std::vector<int> moff(W.nsys);
    size_t tot = 0;
    for (int s = 0; s < W.nsys; s++) { moff[s] = (int)tot; tot += (size_t)W.natoms[s] * ((W.natoms[s] + 31) / 32); }
    if (tot > (size_t)INT32_MAX) return fail("exclusion rows too large (%zu words)", tot);
    std::vector<uint32_t> m(tot, 0u);
    for (int s = 0; s < W.nsys; s++) {
        const int na = W.natoms[s], nn = W.nnode[s], a0 = W.desc[s].x, n0 = W.desc[s].y, nb = (na + 31) / 32;
        uint32_t* row = m.data() + moff[s];
        auto set = [&](int i, int j) { row[i * nb + (j >> 5)] |= 1u << (j & 31); };
        for (int i = 0; i < na; i++) {
            set(i, i);
            for (int j = na; j < 32 * nb; j++) set(i, j);
            const int4 g = W.h_ng[a0 + i], c = W.h_ngC[a0 + i];
            const int gg[4] = {g.x, g.y, g.z, g.w}, cc[4] = {c.x, c.y, c.z, c.w};
            for (int k = 0; k < 4; k++)
                if (gg[k] >= 0 && (!pbc || cc[k] == central)) { set(i, gg[k]); set(gg[k], i); }
        }
        if (!x13) continue;
        for (int ia = 0; ia < nn; ia++) {
            const int bits = W.h_a13[n0 + ia];
            if (!bits) continue;
            const int4 g = W.h_ng[a0 + ia], c = W.h_ngC[a0 + ia];
            const int gg[4] = {g.x, g.y, g.z, g.w}, cc[4] = {c.x, c.y, c.z, c.w};
            for (int i = 0; i < 3; i++) for (int j = i + 1; j < 4; j++)
                if (((bits >> angle_slot(i, j)) & 1) && (!pbc || cc[i] == cc[j])) { set(gg[i], gg[j]); set(gg[j], gg[i]); }
        }
    }
    if (upload(W.d_moff, moff) || upload(W.d_xmask, m)) return -1;
    CK(cudaStreamSynchronize(W.stream));
    return 0;
}

int build_buckets() {
    for (auto& B : W.buckets) { B.queue.release(); B.vl.release(); }
    W.buckets.clear();
    W.graph_valid = false;
    std::vector<std::vector<int>> groups(6);
    for (int s = 0; s < W.nsys; s++) groups[size_class(W.natoms[s])].push_back(s);
    // largest systems first: their buckets are launched first
    for (int k = 5; k >= 0; k--) {
        if (groups[k].empty()) continue;
        Bucket B;
        B.sys = groups[k];
        std::stable_sort(B.sys.begin(), B.sys.end(), [](int a, int b) { return W.natoms[a] > W.natoms[b]; });
        int maxNA = 0;
        for (int s : B.sys) maxNA = std::max(maxNA, W.natoms[s]);
        int kind, apl, T, S;
        default_config(k, maxNA, kind, apl, T, S);
        const Tune& tu = W.tune[k];
        if (tu.kind >= 0 && !W.force_T && !W.force_S) { kind = tu.kind; apl = tu.apl; T = tu.T; S = tu.S; }
        if (config_bucket(B, kind, apl, T, S)) return -1;
        B.cls = k;
        W.buckets.push_back(std::move(B));
    }
    while (W.bstreams.size() < W.buckets.size()) {
        cudaStream_t s; CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); W.bstreams.push_back(s);
        cudaEvent_t e; CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)); W.bev.push_back(e);
    }
    if (build_xmask()) return -1;
    W.buckets_dirty = false;
    return 0;
}

// Page-locked host staging for the per-call state copies (positions and
// velocities in, state out), so the transfers run at full PCIe/C2C rate.
struct PinnedBuf {
    float4* p = nullptr; size_t n = 0;
    int ensure(size_t cnt) {
        if (cnt <= n && p) return 0;
        if (p) cudaFreeHost(p);
        p = nullptr; n = 0;
        if (cudaHostAlloc(reinterpret_cast<void**>(&p), cnt * sizeof(float4), cudaHostAllocDefault) != cudaSuccess)
            return fail("cudaHostAlloc(%zu B) failed", cnt * sizeof(float4));
        n = cnt;
        return 0;
    }
};
PinnedBuf g_stage_a, g_stage_b;


// the bucket's pair-list scratch into the launch parameters (CTA relax kernels)
void set_lists(Params& P, const Bucket& B) {
    const bool on = W.pair_lists && B.kind == 0 && B.vstride > 4 * B.maxNA && B.vl.p;
    P.vlist = on ? B.vl.p : nullptr;
    P.vstride = on ? B.vstride : 0;
    P.vcap = on ? B.vstride - 4 * B.maxNA : 0;
    P.vskin = (float)W.list_skin;
}

// the launches of one relax call on the library stream: reset the work
// counters, fork to one stream per bucket, one persistent kernel per bucket
// (systems claimed through the bucket's queue), join
int enqueue_relax(const Params& P) {
    Params Pc = P;
    Systems Y = make_systems();
    CK(cudaMemsetAsync(W.d_counter.p, 0, 64 * sizeof(int), W.stream));
    CK(cudaEventRecord(W.evfork, W.stream));
    for (size_t b = 0; b < W.buckets.size(); b++) {
        Bucket& B = W.buckets[b];
        cudaStream_t st = W.bstreams[b];
        CK(cudaStreamWaitEvent(st, W.evfork, 0));
        void* fn = P.md_mode == 2 ? (B.kind ? relax_warp_explore_fn(B.apl) : relax_explore_fn(B.T))
                                  : (B.kind ? relax_warp_fn(B.apl, W.count) : relax_fn(B.T, B.S, W.count));
        const int* q = B.queue.p;
        int nq = (int)B.sys.size();
        int* ctr = W.d_counter.p + b;
        int mna = B.maxNA, mnn = B.maxNN;
        set_lists(Pc, B);
        void* args[] = {&Pc, &Y, &q, &nq, &ctr, &mna, &mnn};
        CK(cudaLaunchKernel(fn, dim3(B.grid), dim3(B.T), args, B.smem, st));
        if (!g_capturing) g_launches++;
    }
    for (size_t b = 0; b < W.buckets.size(); b++) {
        CK(cudaEventRecord(W.bev[b], W.bstreams[b]));
        CK(cudaStreamWaitEvent(W.stream, W.bev[b], 0));
    }
    CK(cudaGetLastError());
    return 0;
}

}  // namespace

void mmff_set_error(const char* msg) { g_err = msg; }
void mmff_count_launches(int n) { g_launches += (unsigned long long)n; }

namespace mmff {

cudaStream_t world_stream() { return ensure_ready() ? nullptr : W.stream; }

int world_view(WorldView* v) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (W.buckets_dirty && build_buckets()) return -1;     // exclusion rows of the current systems
    v->P = make_params(true, 0, 0.0, 0);
    v->Y = make_systems();
    v->stream = W.stream;
    v->nsys = W.nsys; v->NA = W.NA; v->NV = W.NV;
    v->desc = W.desc.data();
    for (int k = 0; k < 3; k++) v->gpos0[k] = W.gpos0[k];
    return 0;
}

}  // namespace mmff

// ============================================================================ C-ABI
extern "C" {

const char* mmff_last_error(void) { return g_err.c_str(); }

unsigned long long mmff_kernel_launches(void) { return g_launches.load(); }

int mmff_init_device(int device) {
    if (W.ready && W.device == device) return 0;
    W.device = device;
    W.ready = false;
    return ensure_ready();
}

int mmff_sync(void) {
    if (ensure_ready()) return -1;
    CK(cudaStreamSynchronize(W.stream));
    CK(cudaGetLastError());
    return 0;
}

int mmff_set_params(int flags, const int* nPBC, double Rcut, double alphaMorse, double FmaxNonBonded) {
    W.version++;
    W.buckets_dirty = true;     // shared-memory size depends on the image set and the cutoff
    W.flags = flags;
    if (nPBC) for (int k = 0; k < 3; k++) W.npbc[k] = nPBC[k];
    W.Rcut = Rcut;
    W.alphaMorse = alphaMorse;
    W.FmaxNB = FmaxNonBonded;
    return 0;
}

int mmff_set_fire(double dt_max, double dt_min, double damp_max, double finc, double fdec, double falpha,
                  int minLastNeg, double cv_kill, double Flim, int variant) {
    W.version++;
    if (variant != 0 && variant != 1) return fail("FIRE variant must be 0 or 1");
    double f[10] = {dt_max, dt_min, damp_max, finc, fdec, falpha, (double)minLastNeg, cv_kill, Flim, (double)variant};
    memcpy(W.fire, f, sizeof f);
    return 0;
}

// Per-atom GridFF stencil cache of the CTA relax kernels on (default) or off
// (every step gathers the 64 grid coefficients); results are bit-identical.
int mmff_set_grid_cache(int on) {
    W.version++;
    W.gcache = on != 0;
    return clear_grid_cache();
}

int mmff_set_launch(int threads, int pair_split) {
    if (threads && threads != 64 && threads != 128 && threads != 256 && threads != 512) return fail("threads must be 64/128/256/512");
    if (pair_split && pair_split != 1 && pair_split != 2 && pair_split != 4 && pair_split != 8) return fail("pair_split must be 1/2/4/8");
    W.force_T = threads; W.force_S = pair_split; W.buckets_dirty = true;
    return 0;
}

int mmff_grid_upload(int nx, int ny, int nz, const double* pos0, const double* step, const double* coefs) {
    W.version++;
    if (ensure_ready()) return -1;
    if (nx < 4 || ny < 4 || nz < 8) return fail("grid too small (%d,%d,%d)", nx, ny, nz);
    const size_t n = (size_t)nx * ny * nz;
    std::vector<float4> h(n);
    for (size_t i = 0; i < n; i++) h[i] = make_float4((float)coefs[3 * i], (float)coefs[3 * i + 1], (float)coefs[3 * i + 2], 0.f);
    if (W.grid.ensure(n)) return -1;
    CK(cudaMemcpyAsync(W.grid.p, h.data(), n * sizeof(float4), cudaMemcpyHostToDevice, W.stream));
    if (clear_grid_cache()) return -1;
    CK(cudaStreamSynchronize(W.stream));
    W.gn[0] = nx; W.gn[1] = ny; W.gn[2] = nz;
    for (int k = 0; k < 3; k++) { W.gpos0[k] = pos0[k]; W.gstep[k] = step[k]; }
    return 0;
}

int mmff_grid_build(int nsub, const double* spos, const double* sREQ, const double* lvec, const int* nPBC_mors,
                    const int* nPBC_coul, double alphaMorse, int nx, int ny, int nz, const double* pos0,
                    const double* step, double* coefs_out) {
    W.version++;
    if (ensure_ready()) return -1;
    if (nx < 4 || ny < 4 || nz < 8 || nsub < 1) return fail("bad grid build arguments");
    const long ntot = (long)nx * ny * nz;
    std::vector<double4> hq(nsub);
    std::vector<double2> hr(nsub);
    for (int i = 0; i < nsub; i++) {
        hq[i] = make_double4(spos[3 * i], spos[3 * i + 1], spos[3 * i + 2], sREQ[4 * i + 2]);
        hr[i] = make_double2(sREQ[4 * i], sREQ[4 * i + 1]);
    }
    auto shifts = [&](const int* np) {
        std::vector<double3> s;
        for (int iz = -np[2]; iz <= np[2]; iz++) for (int iy = -np[1]; iy <= np[1]; iy++) for (int ix = -np[0]; ix <= np[0]; ix++)
            s.push_back(make_double3(lvec[0] * ix + lvec[3] * iy + lvec[6] * iz, lvec[1] * ix + lvec[4] * iy + lvec[7] * iz,
                                     lvec[2] * ix + lvec[5] * iy + lvec[8] * iz));
        return s;
    };
    std::vector<double3> sm = shifts(nPBC_mors), sc = shifts(nPBC_coul);
    DBuf<double4> dq; DBuf<double2> dr; DBuf<double3> dsm, dsc; DBuf<double> V, work;
    if (dq.ensure(nsub) || dr.ensure(nsub) || dsm.ensure(sm.size()) || dsc.ensure(sc.size()) || V.ensure(3 * ntot)) return -1;
    CK(cudaMemcpy(dq.p, hq.data(), nsub * sizeof(double4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dr.p, hr.data(), nsub * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dsm.p, sm.data(), sm.size() * sizeof(double3), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dsc.p, sc.data(), sc.size() * sizeof(double3), cudaMemcpyHostToDevice));
    const int tb = 128;
    grid_potential_kernel<<<(unsigned)((ntot + tb - 1) / tb), tb, 0, W.stream>>>(
        nx, ny, nz, make_double3(pos0[0], pos0[1], pos0[2]), make_double3(step[0], step[1], step[2]), nsub, dq.p, dr.p,
        dsm.p, (int)sm.size(), dsc.p, (int)sc.size(), alphaMorse, V.p);
    CK(cudaGetLastError());
    // z lines (open), then y and x (periodic)
    const long lz = (long)nx * ny, ly = (long)nx * nz, lx = (long)ny * nz;
    const long wmax = std::max(lz * nz, std::max(ly * 2 * ny, lx * 2 * nx));
    if (work.ensure(wmax)) return -1;
    solve_open_kernel<<<(unsigned)((lz + 127) / 128), 128, 0, W.stream>>>(V.p, lz, nz, nz, 1, 1, 0, work.p);
    solve_periodic_kernel<<<(unsigned)((ly + 127) / 128), 128, 0, W.stream>>>(V.p, ly, ny, (long)ny * nz, nz, nz, 1, work.p);
    solve_periodic_kernel<<<(unsigned)((lx + 127) / 128), 128, 0, W.stream>>>(V.p, lx, nx, 1, (long)ny * nz, 1, 0, work.p);
    CK(cudaGetLastError());
    if (W.grid.ensure(ntot)) return -1;
    pack_grid_kernel<<<(unsigned)((ntot + 255) / 256), 256, 0, W.stream>>>(ntot, V.p, W.grid.p);
    CK(cudaGetLastError());
    if (coefs_out) CK(cudaMemcpyAsync(coefs_out, V.p, 3 * ntot * sizeof(double), cudaMemcpyDeviceToHost, W.stream));
    if (clear_grid_cache()) return -1;
    CK(cudaStreamSynchronize(W.stream));
    W.gn[0] = nx; W.gn[1] = ny; W.gn[2] = nz;
    for (int k = 0; k < 3; k++) { W.gpos0[k] = pos0[k]; W.gstep[k] = step[k]; }
    work.release(); V.release(); dq.release(); dr.release(); dsm.release(); dsc.release();
    return 0;
}

int mmff_systems_upload(int nsys, const int* natoms, const int* nnode, const double* pos, const double* vel,
                        const int* neighs, const int* neighCell, const int* bkneighs, const double* REQs,
                        const double* apars, const double* bLs, const double* bKs, const double* Ksp,
                        const double* Kpp, const double* lvec) {
    if (ensure_ready()) return -1;
    if (nsys < 1) return fail("nsys must be >= 1");
    W.nsys = nsys;
    W.natoms.assign(natoms, natoms + nsys);
    W.nnode.assign(nnode, nnode + nsys);
    W.desc.resize(nsys);
    int NA = 0, NN = 0, NV = 0;
    for (int s = 0; s < nsys; s++) {
        if (natoms[s] < 1 || nnode[s] < 0 || nnode[s] > natoms[s]) return fail("system %d: bad sizes natoms=%d nnode=%d", s, natoms[s], nnode[s]);
        W.desc[s] = make_int4(NA, NN, NV, natoms[s]);
        NA += natoms[s]; NN += nnode[s]; NV += natoms[s] + nnode[s];
    }
    W.NA = NA; W.NN = NN; W.NV = NV;
    // validate topology indices (never hand the kernels an out-of-range index)
    const int np = (2 * W.npbc[0] + 1) * (2 * W.npbc[1] + 1) * (2 * W.npbc[2] + 1);
    for (int s = 0; s < nsys; s++) {
        const int a0 = W.desc[s].x, na = natoms[s], nn = nnode[s];
        for (int i = 0; i < na; i++) for (int k = 0; k < 4; k++) {
            const int j = neighs[4 * (a0 + i) + k], c = neighCell[4 * (a0 + i) + k], b = bkneighs[4 * (a0 + i) + k];
            if (j >= na || j < -1) return fail("system %d atom %d: neighbour %d out of range", s, i, j);
            if (j >= 0 && i < nn && (c < 0 || c >= np) && (W.flags & F_PBC)) return fail("system %d atom %d: neighCell %d out of range", s, i, c);
            if (b >= 4 * nn || b < -1) return fail("system %d atom %d: bkneigh %d out of range", s, i, b);
        }
    }
    W.orig.assign(3 * nsys, 0.0);
    std::vector<float4> hpos(NV), hvel(NV), hREQ(NA), hPLQ(NA), hap(NN), hbL(NN), hbK(NN), hks(NN), hkp(NN), hgorg(nsys);
    std::vector<int4> hng(NA), hngC(NA), hbk(NA);
    std::vector<int> ha13(NN);
    std::vector<float> hlv(9 * nsys);
    std::vector<double4> hfire(nsys);
    const double sqk = std::sqrt(14.3996448915);
    for (int s = 0; s < nsys; s++) {
        const int a0 = W.desc[s].x, n0 = W.desc[s].y, v0 = W.desc[s].z, na = natoms[s], nn = nnode[s];
        double c[3] = {0, 0, 0};
        for (int i = 0; i < na; i++) for (int k = 0; k < 3; k++) c[k] += pos[3 * (v0 + i) + k];
        for (int k = 0; k < 3; k++) { c[k] /= na; W.orig[3 * s + k] = c[k]; }
        for (int i = 0; i < na + nn; i++) {
            const double* p = pos + 3 * (v0 + i);
            if (i < na) hpos[v0 + i] = make_float4((float)(p[0] - c[0]), (float)(p[1] - c[1]), (float)(p[2] - c[2]), 0.f);
            else        hpos[v0 + i] = make_float4((float)p[0], (float)p[1], (float)p[2], 0.f);
            const double* v = vel ? vel + 3 * (v0 + i) : nullptr;
            hvel[v0 + i] = v ? make_float4((float)v[0], (float)v[1], (float)v[2], 0.f) : make_float4(0, 0, 0, 0);
        }
        for (int i = 0; i < na; i++) {
            const double* R = REQs + 4 * (a0 + i);
            hREQ[a0 + i] = make_float4((float)R[0], (float)R[1], (float)(R[2] * sqk), (float)R[3]);
            // Forces.h:611 REQ2PLQ_d
            const double e = std::exp(W.alphaMorse * R[0]);
            const double cL = e * R[1], cP = e * cL;
            hPLQ[a0 + i] = make_float4((float)cP, (float)cL, (float)R[2], (float)(e * e * R[3]));
            const int* g = neighs + 4 * (a0 + i); hng[a0 + i] = make_int4(g[0], g[1], g[2], g[3]);
            const int* gc = neighCell + 4 * (a0 + i); hngC[a0 + i] = make_int4(gc[0], gc[1], gc[2], gc[3]);
            const int* b = bkneighs + 4 * (a0 + i); hbk[a0 + i] = make_int4(b[0], b[1], b[2], b[3]);
        }
        for (int i = 0; i < nn; i++) {
            auto f4 = [&](const double* a) { return make_float4((float)a[4 * (n0 + i)], (float)a[4 * (n0 + i) + 1], (float)a[4 * (n0 + i) + 2], (float)a[4 * (n0 + i) + 3]); };
            hap[n0 + i] = f4(apars); hbL[n0 + i] = f4(bLs); hbK[n0 + i] = f4(bKs); hks[n0 + i] = f4(Ksp); hkp[n0 + i] = f4(Kpp);
        }
        angle_pairs13(na, nn, &hng[a0], &ha13[n0]);
        for (int k = 0; k < 9; k++) hlv[9 * s + k] = (float)lvec[9 * s + k];
        hgorg[s] = make_float4((float)(c[0] - W.gpos0[0]), (float)(c[1] - W.gpos0[1]), (float)(c[2] - W.gpos0[2]), 0.f);
        hfire[s] = make_double4(W.fire[0], W.fire[2], 0.0, 0.0);
    }
    std::vector<int4> hdesc = W.desc;
    if (upload(W.d_desc, hdesc) || upload(W.d_nnode, W.nnode) || upload(W.d_lvec, hlv) || upload(W.d_gorg, hgorg) ||
        upload(W.d_REQ, hREQ) || upload(W.d_PLQ, hPLQ) || upload(W.d_ng, hng) || upload(W.d_ngC, hngC) ||
        upload(W.d_bk, hbk) || upload(W.d_apar, hap) || upload(W.d_bL, hbL) || upload(W.d_bK, hbK) ||
        upload(W.d_ksp, hks) || upload(W.d_kpp, hkp) || upload(W.d_pos, hpos) || upload(W.d_vel, hvel) ||
        upload(W.d_pos0, hpos) || upload(W.d_vel0, hvel) || upload(W.d_fire, hfire) || upload(W.d_fire0, hfire) ||
        upload(W.d_a13, ha13))
        return -1;
    W.h_ng = std::move(hng); W.h_ngC = std::move(hngC); W.h_a13 = std::move(ha13);
    W.has_constr = false;           // springs belong to the systems they were set for
    W.ndcon = 0; W.nacon = 0;       // and so do the distance / angle constraints
    W.n_explore = -1;               // and the state of the exploring cycle
    if (W.d_force.ensure(NV) || W.d_energy.ensure(nsys) || W.d_status.ensure(nsys) || W.d_nsteps.ensure(nsys) ||
        W.d_fconv.ensure(nsys) || W.d_counter.ensure(64) || W.d_stats.ensure(8) || W.d_gkey.ensure(NA) ||
        W.d_gcs.ensure((size_t)NA * 16) || clear_grid_cache())
        return -1;
    CK(cudaMemsetAsync(W.d_status.p, 0, nsys * sizeof(int), W.stream));
    CK(cudaMemsetAsync(W.d_nsteps.p, 0, nsys * sizeof(int), W.stream));
    CK(cudaStreamSynchronize(W.stream));
    W.buckets_dirty = true;
    return 0;
}

// Position springs of the uploaded systems (relax_multi.cl:995-1010): per atom
// anchor [sum natoms][4] = (x, y, z) in world coordinates and w > 0 to switch
// the spring on, constants K [sum natoms][4] = (kx, ky, kz, -); the relax
// kernels add (anchor - p) * max(K, 0) to the atom's force after the clamp.
// NULL anchor clears them.  Uploading systems clears them too.
int mmff_set_constraints(const double* anchor, const double* K) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    W.version++;
    if (!anchor) { W.has_constr = false; return 0; }
    if (!K) return fail("mmff_set_constraints: K is NULL");
    std::vector<float4> ha(W.NA), hk(W.NA);
    bool any = false;
    for (int s = 0; s < W.nsys; s++) {
        const int a0 = W.desc[s].x;
        const double* o = W.orig.data() + 3 * s;
        for (int i = 0; i < W.natoms[s]; i++) {
            const double* c = anchor + 4 * (a0 + i);
            const double* k = K + 4 * (a0 + i);
            ha[a0 + i] = make_float4((float)(c[0] - o[0]), (float)(c[1] - o[1]), (float)(c[2] - o[2]), c[3] > 0 ? 1.f : -1.f);
            hk[a0 + i] = make_float4((float)k[0], (float)k[1], (float)k[2], 0.f);
            any |= c[3] > 0;
        }
    }
    if (upload(W.d_constr, ha) || upload(W.d_constrK, hk)) return -1;
    CK(cudaStreamSynchronize(W.stream));
    W.has_constr = any;
    return 0;
}

// Distance and angle constraints between atoms (FireCore's Constrains bonds /
// angles, constrains.h), for the relax kernels.  dist_idx [ndist*3] = (system
// or -1 for every system, i0, i1); dist_par [ndist*8] = (lmin, lmax, kmin,
// kmax, flim, shift along a, b, c); ang_idx [nang*4] = (system or -1, centre,
// end 1, end 2); ang_par [nang*2] = (ang0 [rad], k).  Local atom indices.
int mmff_set_bond_constraints(int ndist, const int* dist_idx, const double* dist_par, int nang, const int* ang_idx,
                              const double* ang_par) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (ndist < 0 || nang < 0 || (ndist && (!dist_idx || !dist_par)) || (nang && (!ang_idx || !ang_par)))
        return fail("mmff_set_bond_constraints: bad counts or NULL arrays");
    auto check = [&](int sys, const int* at, int n, const char* what) -> int {
        if (sys < -1 || sys >= W.nsys) return fail("%s constraint: system %d out of range", what, sys);
        for (int k = 0; k < n; k++) {
            const int lim = sys >= 0 ? W.natoms[sys] : *std::min_element(W.natoms.begin(), W.natoms.end());
            if (at[k] < 0 || at[k] >= lim) return fail("%s constraint: atom %d out of range", what, at[k]);
        }
        return 0;
    };
    std::vector<int4> di(ndist), ai(nang);
    std::vector<float4> da(ndist), db(ndist), aa(nang);
    for (int c = 0; c < ndist; c++) {
        const int* x = dist_idx + 3 * c;
        const double* q = dist_par + 8 * c;
        if (check(x[0], x + 1, 2, "distance")) return -1;
        di[c] = make_int4(x[0], x[1], x[2], 0);
        da[c] = make_float4((float)q[1], (float)q[0], (float)q[3], (float)q[2]);   // (lmax, lmin, kmax, kmin)
        db[c] = make_float4((float)q[5], (float)q[6], (float)q[7], (float)q[4]);
    }
    for (int c = 0; c < nang; c++) {
        const int* x = ang_idx + 4 * c;
        const double* q = ang_par + 2 * c;
        if (check(x[0], x + 1, 3, "angle")) return -1;
        ai[c] = make_int4(x[0], x[1], x[2], x[3]);
        aa[c] = make_float4((float)cos(q[0] * 0.5), (float)sin(q[0] * 0.5), (float)q[1], 0.f);
    }
    W.version++;
    W.ndcon = 0; W.nacon = 0;
    if (ndist && (upload(W.d_dci, di) || upload(W.d_dca, da) || upload(W.d_dcb, db))) return -1;
    if (nang && (upload(W.d_aci, ai) || upload(W.d_aca, aa))) return -1;
    CK(cudaStreamSynchronize(W.stream));
    W.ndcon = ndist; W.nacon = nang;
    return 0;
}

// Shifted-image pair lists of the CTA relax kernels on (1, default) or off (0):
// off evaluates the candidate tiles of the shifted images every step.
// skin > 0 sets the list skin [A] (default 1).
int mmff_set_pair_lists(int on, double skin) {
    if (ensure_ready()) return -1;
    if (skin > 0) {
        if (skin > 5.0) return fail("mmff_set_pair_lists: skin %g A out of range (0, 5]", skin);
        W.list_skin = skin;
    }
    W.pair_lists = on != 0;
    W.version++;
    return 0;
}

// Restore positions, velocities and FIRE state from the copy kept at upload (device to device).
int mmff_systems_restore(void) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    CK(cudaMemcpyAsync(W.d_pos.p, W.d_pos0.p, W.NV * sizeof(float4), cudaMemcpyDeviceToDevice, W.stream));
    CK(cudaMemcpyAsync(W.d_vel.p, W.d_vel0.p, W.NV * sizeof(float4), cudaMemcpyDeviceToDevice, W.stream));
    CK(cudaMemcpyAsync(W.d_fire.p, W.d_fire0.p, W.nsys * sizeof(double4), cudaMemcpyDeviceToDevice, W.stream));
    CK(cudaMemsetAsync(W.d_status.p, 0, W.nsys * sizeof(int), W.stream));
    return 0;
}

// Overwrite positions (and velocities, or zero them) of all systems; FIRE state reset.
int mmff_systems_set_state(const double* pos, const double* vel, int reset_fire) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (g_stage_a.ensure(W.NV) || g_stage_b.ensure(W.NV)) return -1;
    float4* hpos = g_stage_a.p;
    float4* hvel = g_stage_b.p;
    for (int s = 0; s < W.nsys; s++) {
        const int v0 = W.desc[s].z, na = W.natoms[s], nn = W.nnode[s];
        const double* c = W.orig.data() + 3 * s;
        for (int i = 0; i < na + nn; i++) {
            const double* p = pos + 3 * (v0 + i);
            hpos[v0 + i] = (i < na) ? make_float4((float)(p[0] - c[0]), (float)(p[1] - c[1]), (float)(p[2] - c[2]), 0.f)
                                    : make_float4((float)p[0], (float)p[1], (float)p[2], 0.f);
            const double* v = vel ? vel + 3 * (v0 + i) : nullptr;
            hvel[v0 + i] = v ? make_float4((float)v[0], (float)v[1], (float)v[2], 0.f) : make_float4(0, 0, 0, 0);
        }
    }
    CK(cudaMemcpyAsync(W.d_pos.p, hpos, W.NV * sizeof(float4), cudaMemcpyHostToDevice, W.stream));
    CK(cudaMemcpyAsync(W.d_vel.p, hvel, W.NV * sizeof(float4), cudaMemcpyHostToDevice, W.stream));
    if (reset_fire) {
        std::vector<double4> hf(W.nsys, make_double4(W.fire[0], W.fire[2], 0.0, 0.0));
        CK(cudaMemcpyAsync(W.d_fire.p, hf.data(), W.nsys * sizeof(double4), cudaMemcpyHostToDevice, W.stream));
    }
    CK(cudaStreamSynchronize(W.stream));
    return 0;
}

int mmff_eval(int with_energy) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (W.buckets_dirty && build_buckets()) return -1;
    Params P = make_params(true, 0, 0.0, 0);
    Systems Y = make_systems();
    for (auto& B : W.buckets) {
        void* fn = B.kind ? eval_warp_fn(B.apl, with_energy != 0) : eval_fn(B.T, B.S, with_energy != 0);
        const int* q = B.queue.p;
        int nq = (int)B.sys.size();
        int mna = B.maxNA, mnn = B.maxNN;
        void* args[] = {&P, &Y, &q, &nq, &mna, &mnn};
        const int nblk = B.kind ? (nq + 3) / 4 : nq;
        CK(cudaLaunchKernel(fn, dim3(nblk), dim3(B.T), args, B.smem, W.stream));
        g_launches++;
    }
    CK(cudaGetLastError());
    return 0;
}

// Relax every system for up to nstep_max FIRE steps (persistent, one launch per
// size bucket, buckets run concurrently on their own streams).
int mmff_relax(int nstep_max, double Fconv, int conv_mode) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (W.buckets_dirty && build_buckets()) return -1;
    Params P = make_params(false, nstep_max, Fconv, conv_mode);
    if (!W.use_graph) return enqueue_relax(P);
    // one CUDA graph per (parameters, step limit, criterion): the counter reset,
    // the fork to the bucket streams, every bucket's persistent kernel and the join
    const bool same = W.graph_valid && W.gkey_nstep == nstep_max && W.gkey_fconv == Fconv &&
                      W.gkey_mode == conv_mode && W.gkey_count == W.count && W.gkey_version == W.version;
    if (!same) {
        if (W.gexec) { cudaGraphExecDestroy(W.gexec); W.gexec = nullptr; }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(W.stream, cudaStreamCaptureModeThreadLocal));
        g_capturing = true;
        const int rc = enqueue_relax(P);
        g_capturing = false;
        const cudaError_t e = cudaStreamEndCapture(W.stream, &g);
        if (rc) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return -1; }
        if (e != cudaSuccess) return fail("relax graph capture: %s", cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&W.gexec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) { W.gexec = nullptr; return fail("relax graph instantiate: %s", cudaGetErrorString(ei)); }
        W.graph_valid = true; W.gkey_nstep = nstep_max; W.gkey_fconv = Fconv; W.gkey_mode = conv_mode;
        W.gkey_count = W.count; W.gkey_version = W.version;
    }
    CK(cudaGraphLaunch(W.gexec, W.stream));
    g_launches += W.buckets.size();
    return 0;
}

// Substrate atoms for the direct term (flag F_SURF): positions [nsub][3] in
// world coordinates, REQ [nsub][4] = (R0, sqrt(E0), Q, H), lattice vectors
// [9] and image counts [3] of the substrate, Coulomb damping radius Rdamp.
int mmff_surf_upload(int nsub, const double* spos, const double* sREQ, const double* lvec, const int* nPBC,
                     double Rdamp) {
    if (ensure_ready()) return -1;
    if (nsub < 0 || (nsub > 0 && (!spos || !sREQ || !lvec || !nPBC))) return fail("mmff_surf_upload: bad arguments");
    const double sqke = sqrt(14.3996448915);    // Coulomb constant [eV A / e^2], folded into the charges
    std::vector<float4> hp(nsub), hr(nsub);
    for (int i = 0; i < nsub; i++) {
        hp[i] = make_float4((float)spos[3 * i], (float)spos[3 * i + 1], (float)spos[3 * i + 2], 0.f);
        hr[i] = make_float4((float)sREQ[4 * i], (float)sREQ[4 * i + 1], (float)(sREQ[4 * i + 2] * sqke), (float)sREQ[4 * i + 3]);
    }
    if (upload(W.d_spos, hp) || upload(W.d_sREQ, hr)) return -1;
    CK(cudaStreamSynchronize(W.stream));
    W.nsurf = nsub;
    for (int k = 0; k < 3; k++) W.snpbc[k] = nPBC ? nPBC[k] : 0;
    for (int k = 0; k < 9; k++) W.slv[k] = lvec ? (float)lvec[k] : 0.f;
    W.sRdamp = Rdamp;
    W.version++;
    return 0;
}

// Langevin drive parameters (MMFFsp3_loc::move_atom_Langevin): time step,
// friction gamma, temperature T [K], random-stream seed (resets the step count).
int mmff_set_md(double dt, double gamma, double T, unsigned long long seed) {
    if (!(dt > 0) || gamma < 0 || T < 0) return fail("mmff_set_md: need dt > 0, gamma >= 0, T >= 0");
    W.md_dt = dt; W.md_gamma = gamma; W.md_T = T; W.md_seed = seed; W.md_step = 0;
    return 0;
}

// nsteps Langevin steps for every system (same persistent kernels as relax,
// FIRE replaced by the drive; forces clamped by Flim when set).  Asynchronous.
int mmff_md(int nsteps) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (nsteps < 0) return fail("mmff_md: nsteps must be >= 0");
    if (W.buckets_dirty && build_buckets()) return -1;
    Params P = make_params(false, nsteps, -1.0, 1);
    const double kB = 8.617333262e-5;     // eV/K (const_kB)
    P.md_mode = 1;
    P.md_dt = (float)W.md_dt;
    P.md_gamma = (float)W.md_gamma;
    P.md_noise = (float)sqrt(2.0 * kB * W.md_T * W.md_gamma / W.md_dt);
    P.md_seed = W.md_seed;
    P.md_step0 = W.md_step;
    if (enqueue_relax(P)) return -1;
    W.md_step += nsteps;
    return 0;
}

// Exploring cycle of the global optimiser (GOpt.h:25-60 with
// MolWorld_sp3_multi.h:770-833 and MolWorld_sp3.h:2290-2296,2397-2473): every
// system relaxes with FIRE; a minimum (convergence measure below Fconv) is
// kept and starts an exploring phase of Langevin steps (mmff_set_md's dt,
// gamma, T and random stream); a FIRE phase longer than n_relax steps
// (n_relax <= 0: never) is given up and starts one too; an exploring phase
// ends after n_explore steps.  Resets the cycle's per-system state: exploring
// (start_exploring != 0) or relaxing, no minima found yet, the kept minimum =
// the current positions.  Uploading systems clears it.
int mmff_set_explore(int n_explore, int n_relax, int start_exploring) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (n_explore < 0) return fail("mmff_set_explore: n_explore must be >= 0");
    if (W.d_gopt.ensure(W.nsys) || W.d_minpos.ensure(W.NV)) return -1;
    std::vector<int4> h(W.nsys, make_int4(start_exploring ? 1 : 0, 0, 0, 0));
    if (upload(W.d_gopt, h)) return -1;
    CK(cudaMemcpyAsync(W.d_minpos.p, W.d_pos.p, W.NV * sizeof(float4), cudaMemcpyDeviceToDevice, W.stream));
    CK(cudaStreamSynchronize(W.stream));
    W.n_explore = n_explore;
    W.n_relax = n_relax;
    return 0;
}

// nsteps steps of the exploring cycle for every system (same persistent
// kernels as relax; no system retires, so every system runs nsteps steps;
// convergence measure as mmff_relax's conv_mode).  Asynchronous.
int mmff_explore(int nsteps, double Fconv, int conv_mode) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (W.n_explore < 0) return fail("mmff_explore: call mmff_set_explore for the current systems first");
    if (nsteps < 0) return fail("mmff_explore: nsteps must be >= 0");
    if (W.buckets_dirty && build_buckets()) return -1;
    Params P = make_params(false, nsteps, Fconv, conv_mode);
    const double kB = 8.617333262e-5;     // eV/K (const_kB)
    P.md_mode = 2;
    P.md_dt = (float)W.md_dt;
    P.md_gamma = (float)W.md_gamma;
    P.md_noise = (float)sqrt(2.0 * kB * W.md_T * W.md_gamma / W.md_dt);
    P.md_seed = W.md_seed;
    P.md_step0 = W.md_step;
    P.n_explore = W.n_explore;
    P.n_relax = W.n_relax;
    if (enqueue_relax(P)) return -1;
    W.md_step += nsteps;
    return 0;
}

// State of the exploring cycle: gopt [nsys][4] = (exploring, steps in the
// current phase, minima found, relax phases given up); minpos (nullable)
// [sum(natoms+nnode)][3] = the last minimum found per system, in world
// coordinates like mmff_get_state's positions (the positions of
// mmff_set_explore's call where none was found yet).
int mmff_get_explore(int* gopt, double* minpos) {
    if (mmff_sync()) return -1;
    if (W.n_explore < 0) return fail("mmff_get_explore: no exploring cycle set up for the current systems");
    if (gopt) CK(cudaMemcpy(gopt, W.d_gopt.p, W.nsys * sizeof(int4), cudaMemcpyDeviceToHost));
    if (minpos) {
        std::vector<float4> h(W.NV);
        CK(cudaMemcpy(h.data(), W.d_minpos.p, W.NV * sizeof(float4), cudaMemcpyDeviceToHost));
        for (int s = 0; s < W.nsys; s++) {
            const int v0 = W.desc[s].z, na = W.natoms[s], nn = W.nnode[s];
            const double* c = W.orig.data() + 3 * s;
            for (int i = 0; i < na + nn; i++) {
                const float4 p = h[v0 + i];
                const double sh = i < na ? 1.0 : 0.0;
                minpos[3 * (v0 + i)] = sh * c[0] + p.x;
                minpos[3 * (v0 + i) + 1] = sh * c[1] + p.y;
                minpos[3 * (v0 + i) + 2] = sh * c[2] + p.z;
            }
        }
    }
    return 0;
}

// Relax through a captured CUDA graph (on != 0) or direct launches.
int mmff_set_graph(int on) {
    W.use_graph = on != 0;
    return 0;
}

// ---------------------------------------------------------------- autotuner
namespace {
struct Cand { int kind, apl, T, S; };
std::vector<Cand> candidates(int cls) {
    switch (cls) {
        case 0: return {{1, 1, 128, 1}, {0, 1, 64, 1}, {0, 1, 64, 2}, {0, 1, 64, 4}, {0, 1, 128, 2}, {0, 1, 128, 4}};
        case 1: return {{1, 2, 128, 1}, {0, 1, 64, 1}, {0, 1, 64, 2}, {0, 1, 128, 1}, {0, 1, 128, 2}, {0, 1, 128, 4}};
        case 3: return {{0, 1, 64, 1}, {0, 1, 64, 2}, {0, 1, 128, 1}, {0, 1, 128, 2}, {0, 1, 128, 4}, {0, 1, 256, 2}, {0, 1, 256, 4}};
        case 4: return {{0, 1, 128, 1}, {0, 1, 128, 2}, {0, 1, 256, 1}, {0, 1, 256, 2}, {0, 1, 512, 1}, {0, 1, 512, 2}};
        case 5: return {{0, 1, 256, 1}, {0, 1, 256, 2}, {0, 1, 512, 1}, {0, 1, 512, 2}, {0, 1, 512, 4}};
        default: return {};
    }
}
}  // namespace

// Time every candidate launch configuration of each size class present on a
// sample of that class's systems (nstep_probe FIRE steps, no convergence
// exit) and keep the fastest for later relax/eval calls.  Positions,
// velocities and FIRE state are restored afterwards.  report (nullable):
// 6 floats per candidate tried (class, kind, atoms per lane, threads, pair
// lanes, microseconds per system-step; negative: not launchable).
int mmff_autotune(int nstep_probe, int max_sample, float* report, int report_cap) {
    if (ensure_ready()) return -1;
    if (!W.nsys) return fail("no systems uploaded");
    if (nstep_probe < 1 || max_sample < 1) return fail("autotune: nstep_probe and max_sample must be >= 1");
    if (W.force_T || W.force_S) return fail("autotune: clear mmff_set_launch overrides first");
    // the candidate kernels read the exclusion rows of the current systems
    if (W.buckets_dirty && build_buckets()) return -1;
    DBuf<float4> sp, sv; DBuf<double4> sf; DBuf<int> sst, sns; DBuf<float> sfc;
    if (sp.ensure(W.NV) || sv.ensure(W.NV) || sf.ensure(W.nsys) || sst.ensure(W.nsys) || sns.ensure(W.nsys) ||
        sfc.ensure(W.nsys))
        return -1;
    auto copy_state = [&](bool save) -> int {
        auto cp = [&](void* a, void* b, size_t n) { return cudaMemcpyAsync(save ? a : b, save ? b : a, n, cudaMemcpyDeviceToDevice, W.stream); };
        CK(cp(sp.p, W.d_pos.p, W.NV * sizeof(float4)));
        CK(cp(sv.p, W.d_vel.p, W.NV * sizeof(float4)));
        CK(cp(sf.p, W.d_fire.p, W.nsys * sizeof(double4)));
        CK(cp(sst.p, W.d_status.p, W.nsys * sizeof(int)));
        CK(cp(sns.p, W.d_nsteps.p, W.nsys * sizeof(int)));
        CK(cp(sfc.p, W.d_fconv.p, W.nsys * sizeof(float)));
        return 0;
    };
    if (copy_state(true)) return -1;
    std::vector<std::vector<int>> groups(6);
    for (int s = 0; s < W.nsys; s++) groups[size_class(W.natoms[s])].push_back(s);
    Params P = make_params(false, nstep_probe, 0.0, 1);     // Fmax < 0: never converges
    Systems Y = make_systems();
    int nrep = 0;
    for (int cls = 0; cls < 6; cls++) {
        std::vector<int>& g = groups[cls];
        if (g.empty()) continue;
        std::stable_sort(g.begin(), g.end(), [](int a, int b) { return W.natoms[a] > W.natoms[b]; });
        std::vector<int> sample;
        const int ns = std::min<int>(max_sample, (int)g.size());
        for (int i = 0; i < ns; i++) sample.push_back(g[(size_t)i * g.size() / ns]);
        float best = 1e30f;
        Tune bt;
        for (const Cand& c : candidates(cls)) {
            Bucket B;
            B.sys = sample;
            float us = -1.f;
            if (config_bucket(B, c.kind, c.apl, c.T, c.S) == 0) {
                void* fn = B.kind ? relax_warp_fn(B.apl, false) : relax_fn(B.T, B.S, false);
                const int* q = B.queue.p;
                int nq = (int)B.sys.size(), mna = B.maxNA, mnn = B.maxNN;
                int* ctr = W.d_counter.p + 32;
                set_lists(P, B);
                void* args[] = {&P, &Y, &q, &nq, &ctr, &mna, &mnn};
                float ms = 0.f;
                for (int rep = 0; rep < 2; rep++) {        // first launch warms caches and clocks
                    if (copy_state(false)) return -1;
                    CK(cudaMemsetAsync(ctr, 0, sizeof(int), W.stream));
                    CK(cudaEventRecord(W.ev0, W.stream));
                    CK(cudaLaunchKernel(fn, dim3(B.grid), dim3(B.T), args, B.smem, W.stream));
                    g_launches++;
                    CK(cudaEventRecord(W.ev1, W.stream));
                    CK(cudaEventSynchronize(W.ev1));
                    CK(cudaEventElapsedTime(&ms, W.ev0, W.ev1));
                }
                us = 1e3f * ms / ((float)ns * (float)nstep_probe);
                if (us < best) { best = us; bt.kind = c.kind; bt.apl = c.apl; bt.T = c.T; bt.S = c.S; bt.us_per_sys_step = us; }
            } else {
                cudaGetLastError();
            }
            B.queue.release();
            B.vl.release();
            if (report && nrep < report_cap) {
                const float row[6] = {(float)cls, (float)c.kind, (float)c.apl, (float)c.T, (float)c.S, us};
                for (int j = 0; j < 6; j++) report[6 * nrep + j] = row[j];
            }
            nrep++;
        }
        if (bt.kind >= 0) W.tune[cls] = bt;
    }
    if (copy_state(false)) return -1;
    CK(cudaStreamSynchronize(W.stream));
    W.buckets_dirty = true;
    g_err.clear();
    return nrep;
}

// Tuned configuration of a size class: out = (kind, atoms per lane, threads,
// pair lanes); kind -1 = heuristic.  Set it back (e.g. from a saved file).
int mmff_get_tuning(int cls, int* out) {
    if (cls < 0 || cls > 5) return fail("size class must be 0..5");
    const Tune& t = W.tune[cls];
    out[0] = t.kind; out[1] = t.apl; out[2] = t.T; out[3] = t.S;
    return 0;
}

int mmff_set_tuning(int cls, int kind, int apl, int T, int S) {
    if (cls < 0 || cls > 5) return fail("size class must be 0..5");
    if (kind == 1 && !((cls == 0 && apl == 1) || (cls == 1 && apl == 2))) return fail("warp engine only for classes 0/1 (apl = class + 1)");
    if (kind == 0 && !relax_fn(T, S, false)) return fail("no CTA kernel with T=%d S=%d", T, S);
    if (kind != -1 && kind != 0 && kind != 1) return fail("kind must be -1, 0 or 1");
    W.tune[cls].kind = kind; W.tune[cls].apl = apl; W.tune[cls].T = T; W.tune[cls].S = S;
    W.buckets_dirty = true;
    return 0;
}

int mmff_get_forces(double* force) {
    if (mmff_sync()) return -1;
    std::vector<float4> h(W.NV);
    CK(cudaMemcpy(h.data(), W.d_force.p, W.NV * sizeof(float4), cudaMemcpyDeviceToHost));
    for (int i = 0; i < W.NV; i++) { force[3 * i] = h[i].x; force[3 * i + 1] = h[i].y; force[3 * i + 2] = h[i].z; }
    return 0;
}

int mmff_get_energies(double* E) {
    if (mmff_sync()) return -1;
    CK(cudaMemcpy(E, W.d_energy.p, W.nsys * sizeof(double4), cudaMemcpyDeviceToHost));
    return 0;
}

int mmff_get_state(double* pos, double* vel, double* fire, int* status, int* nsteps, double* fconv) {
    if (mmff_sync()) return -1;
    if (pos || vel) {
        if (g_stage_a.ensure(W.NV) || g_stage_b.ensure(W.NV)) return -1;
        const float4* hp = g_stage_a.p;
        const float4* hv = g_stage_b.p;
        CK(cudaMemcpyAsync(g_stage_a.p, W.d_pos.p, W.NV * sizeof(float4), cudaMemcpyDeviceToHost, W.stream));
        if (vel) CK(cudaMemcpyAsync(g_stage_b.p, W.d_vel.p, W.NV * sizeof(float4), cudaMemcpyDeviceToHost, W.stream));
        CK(cudaStreamSynchronize(W.stream));
        for (int s = 0; s < W.nsys; s++) {
            const int v0 = W.desc[s].z, na = W.natoms[s], nn = W.nnode[s];
            const double* c = W.orig.data() + 3 * s;
            for (int i = 0; i < na + nn; i++) {
                const float4 p = hp[v0 + i], v = vel ? hv[v0 + i] : make_float4(0.f, 0.f, 0.f, 0.f);
                if (pos) {
                    if (i < na) { pos[3 * (v0 + i)] = c[0] + p.x; pos[3 * (v0 + i) + 1] = c[1] + p.y; pos[3 * (v0 + i) + 2] = c[2] + p.z; }
                    else { pos[3 * (v0 + i)] = p.x; pos[3 * (v0 + i) + 1] = p.y; pos[3 * (v0 + i) + 2] = p.z; }
                }
                if (vel) { vel[3 * (v0 + i)] = v.x; vel[3 * (v0 + i) + 1] = v.y; vel[3 * (v0 + i) + 2] = v.z; }
            }
        }
    }
    if (fire) CK(cudaMemcpy(fire, W.d_fire.p, W.nsys * sizeof(double4), cudaMemcpyDeviceToHost));
    if (status) CK(cudaMemcpy(status, W.d_status.p, W.nsys * sizeof(int), cudaMemcpyDeviceToHost));
    if (nsteps) CK(cudaMemcpy(nsteps, W.d_nsteps.p, W.nsys * sizeof(int), cudaMemcpyDeviceToHost));
    if (fconv) {
        std::vector<float> h(W.nsys);
        CK(cudaMemcpy(h.data(), W.d_fconv.p, W.nsys * sizeof(float), cudaMemcpyDeviceToHost));
        for (int s = 0; s < W.nsys; s++) fconv[s] = h[s];
    }
    return 0;
}

// B-spline sample at n points (absolute coordinates) with per-point PLQ: fe[n*4]
int mmff_grid_sample(int n, const double* pos, const double* PLQ, double* fe) {
    if (ensure_ready()) return -1;
    if (!W.grid.p) return fail("no grid");
    std::vector<float4> hp(n), hq(n), hf(n);
    for (int i = 0; i < n; i++) {
        hp[i] = make_float4((float)(pos[3 * i] - W.gpos0[0]), (float)(pos[3 * i + 1] - W.gpos0[1]), (float)(pos[3 * i + 2] - W.gpos0[2]), 0.f);
        hq[i] = make_float4((float)PLQ[4 * i], (float)PLQ[4 * i + 1], (float)PLQ[4 * i + 2], (float)PLQ[4 * i + 3]);
    }
    DBuf<float4> dp, dq, df;
    if (dp.ensure(n) || dq.ensure(n) || df.ensure(n)) return -1;
    CK(cudaMemcpy(dp.p, hp.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dq.p, hq.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    Params P = make_params(true, 0, 0, 0);
    grid_sample_kernel<<<(unsigned)((4 * n + 127) / 128), 128, 0, W.stream>>>(P, n, dp.p, dq.p, df.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hf.data(), df.p, n * sizeof(float4), cudaMemcpyDeviceToHost, W.stream));
    CK(cudaStreamSynchronize(W.stream));
    for (int i = 0; i < n; i++) { fe[4 * i] = hf[i].x; fe[4 * i + 1] = hf[i].y; fe[4 * i + 2] = hf[i].z; fe[4 * i + 3] = hf[i].w; }
    dp.release(); dq.release(); df.release();
    return 0;
}

// CUDA-event timing on the library stream
int mmff_timer_start(void) {
    if (ensure_ready()) return -1;
    CK(cudaEventRecord(W.ev0, W.stream));
    return 0;
}
double mmff_timer_stop(void) {
    if (cudaEventRecord(W.ev1, W.stream) != cudaSuccess) return -1.0;
    if (cudaEventSynchronize(W.ev1) != cudaSuccess) return -1.0;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, W.ev0, W.ev1) != cudaSuccess) return -1.0;
    return ms;
}

// Counting mode: the relax kernels also count pair-images inside the cutoff,
// atom grid samples and force evaluations (for the roofline's algorithmic work).
int mmff_set_counting(int on) {
    if (ensure_ready()) return -1;
    W.count = on != 0;
    if (W.d_stats.ensure(8)) return -1;
    CK(cudaMemsetAsync(W.d_stats.p, 0, 8 * sizeof(unsigned long long), W.stream));
    return 0;
}
int mmff_get_counters(unsigned long long* out) {
    if (mmff_sync()) return -1;
    CK(cudaMemcpy(out, W.d_stats.p, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return 0;
}

int mmff_num_buckets(void) { return W.buckets_dirty ? -1 : (int)W.buckets.size(); }
int mmff_bucket_info(int b, int* info) {
    if (b < 0 || b >= (int)W.buckets.size()) return fail("bad bucket");
    const Bucket& B = W.buckets[b];
    info[0] = B.T; info[1] = B.kind ? -B.apl : B.S; info[2] = (int)B.sys.size(); info[3] = B.maxNA; info[4] = B.maxNN; info[5] = B.smem; info[6] = B.grid;
    return 0;
}

}  // extern "C"
