// Internal declarations of liblpmgpu: device state of one problem, launch helpers and the
// kernels' entry points.  Everything here is compiled with -fmad=false so that each C
// operator rounds once, as in the reference's own build (-ffp-contract=off): the bond,
// force and stiffness kernels then reproduce the reference's arithmetic bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lpmgpu.h"

namespace lpm
{

constexpr int kMaxBonds = 32;    // bonds per particle supported by the fixed-size staging
constexpr int kMaxConns = 128;   // connections per particle (SC 61, FCC/BCC below 100)
constexpr int kMaxCand = 512;    // connection candidates per particle before sort-unique
constexpr double kEps = 1e-6;    // include/lpm.h:41
constexpr int kSlice = 32;       // rows per slice of the sliced-ELL stiffness layout

// std::max semantics ((a < b) ? b : a), which keeps the first argument when b is NaN
__host__ __device__ inline double std_max(double a, double b) { return (a < b) ? b : a; }

struct Cell
{
    int lattice = 0, dim = 2, nneighbors = 0;
    double radius = 0, cutoff[2] = {0, 0}, pvol = 0;
    double el[9] = {0};
};

// Unit cell constants of include/unit_cell.h:27-122
Cell make_cell(int lattice, double radius);
// setParticleProperty (particle_elastic.h:70-108): Kn/Tv coefficients
void kntv(const Cell &c, int plane_stress, double E, double mu, double out[3]);
// the same from given elastic constants C11, C12, C44 (particle_elastic.h:110-140)
void kntv_cij(const Cell &c, const double Ce[3], double out[3]);

// Reduction scratch: per-block partial sums and the scalars they reduce to.
struct Scalars
{
    double res_sq;        // ||residual||^2 of the last updateRR
    double reaction_sq;   // running in-order-free sum of squares of the reaction history
    double norm_diag;     // ||diag(K)|| before the BC elimination
    double pad;
    int any_flag;         // damage update: some bond broke / damage changed
    int err;              // topology overflow or a timed-out wait
    int pad2[2];
};

// Device state of one problem.  Particles are indexed by id; bonds are owner-major CSR
// (bstart), each particle's layer-0 list first then its layer-1 list, both ascending in the
// partner id (assembly.h:218-229).
//
// The stiffness is full symmetric and stored sliced-ELL: particle rows are ordered by
// descending connection count (stable, so equal counts keep id order) and grouped in slices of
// kSlice rows; in 2D the slices are then reordered whole so that each width is spread evenly
// over the slice order (perm: position -> id).  Slice s holds width(s) = its longest row's count of block
// columns starting at block slot slice_off[s].  Block slot b, entry e = r*d + c (row-major d x d)
// of the row at lane l lives at K[(b*d*d + e)*kSlice + l]; its particle column at
// col_sell[b*kSlice + l].  A row's k-th block is its k-th connection (ascending id).  A warp
// streams 32 rows in lockstep: every matrix load is 256 contiguous bytes and the x gathers of
// interior rows hit 32 consecutive particles.
struct Problem
{
    lpmgpu_desc desc{};
    Cell cell;
    int n = 0, dim = 2, nsv = 1;
    int64_t nbonds = 0, nnzb = 0, nnz_upper = 0;
    int max_bonds = 0, max_conns = 0;
    int max_records = 0; // largest sum over a particle's bonds of the partner's same-layer bond count
    double kntv[3] = {0, 0, 0};
    cudaStream_t stream = nullptr;
    int device = 0, num_sms = 0;

    // particles
    double *xyz = nullptr, *xyz_last = nullptr, *pin = nullptr, *pex = nullptr, *stress = nullptr;
    double *damage = nullptr, *damage_last = nullptr, *damage_visual = nullptr;
    double *ddot_local = nullptr, *sv = nullptr, *sv_last = nullptr;
    int *cons = nullptr, *type = nullptr, *nb = nullptr, *nb0 = nullptr, *bstart = nullptr;
    double *dLe_total = nullptr, *TdLe_total = nullptr, *cs_sum = nullptr;
    // bonds
    int *bp2 = nullptr, *brev = nullptr;
    double *dis0 = nullptr, *dis = nullptr, *dis_last = nullptr, *dLe = nullptr, *dLp = nullptr,
           *dLp_last = nullptr, *bstrain = nullptr, *Kn = nullptr, *Tv = nullptr, *cs = nullptr,
           *bforce = nullptr, *bforce_last = nullptr, *bdamage = nullptr, *bdamage_last = nullptr;
    // nonlocal neighbours (Assembly::searchNonlocalNeighbors; CSR in ascending id) and the
    // nonlocal damage rate; null when no search ran
    int *nlstart = nullptr, *nlist = nullptr;
    int64_t nnl = 0;
    double *ddot_nonlocal = nullptr;
    // connections and matrices
    int *cstart = nullptr, *conns = nullptr, *nlq = nullptr;
    int64_t *kp_ref = nullptr;        // reference K_pointer (n+1)
    int *perm = nullptr, *iperm = nullptr; // sliced-ELL row order: position -> id, id -> position
    int64_t *slice_off = nullptr;     // nslices+1 block-slot offsets
    int *col_sell = nullptr;          // nsb * kSlice particle columns
    int nslices = 0;
    int cg_grid = 0;                  // > 0: blocks per CG launch (lpmgpu_autotune / lpmgpu_set_cg_grid)
    unsigned long long wait_ns = 4000000000ull; // limit of each grid-barrier wait in k_cg (lpmgpu_set_wait_limit_ns)
    int64_t nsb = 0;                  // block slots of the sliced-ELL layout (>= nnzb / kSlice)
    double *K = nullptr;              // nsb * d*d * kSlice
    float *K32 = nullptr;             // mixed precision copy
    double *diag_raw = nullptr;       // n*d unmodified diagonal (for norm_diag)
    // vectors (n*d)
    double *res = nullptr, *x = nullptr, *r = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr;
    float *x32 = nullptr, *r32 = nullptr, *pa32 = nullptr, *pb32 = nullptr, *q32 = nullptr, *b32 = nullptr;
    float *r32b = nullptr, *w32b = nullptr, *s32b = nullptr; // second buffers of the batch's single-reduction CG
    // reductions
    double *partials = nullptr;       // kMaxGridBlocks * 4
    Scalars *scal = nullptr;
    Scalars *scal_host = nullptr;     // pinned mirror
    unsigned *barrier = nullptr;      // [0] count, [1] generation
    int64_t *cg_info = nullptr;       // device CG status words
    int64_t *cg_info_host = nullptr;  // pinned mirror
    // timing
    cudaEvent_t ev[8];
    double phase_s[4] = {0, 0, 0, 0};
    lpmgpu_counters ctr{};
    cudaEvent_t cg_ev[2] = {nullptr, nullptr};
    int64_t device_bytes = 0;
    std::vector<void *> allocs;
    // host copies of the coordinates and types given at creation (Particle::xyz_initial, type)
    // and the per-step dump writer (dump.cu), created by the first lpmgpu_dump_write
    std::vector<double> xyz0_host;
    std::vector<int> type_host;
    void *dump = nullptr;
    // the force-state sequence (geometry + bond forces, particle forces + residual, the scalar
    // record's copy) as CUDA graphs, without / with the reaction accumulation of updateRR;
    // captured at first use, replayed afterwards (graphs_off: capture failed or LPMGPU_NO_GRAPHS)
    cudaGraphExec_t fs_graph[2] = {nullptr, nullptr};
    // Assembly::storeStateVar / resetStateVar(true) (seven copies each) as graphs
    cudaGraphExec_t state_graph[2] = {nullptr, nullptr};
    bool graphs_off = false;
    // K's version, raised by every assembly; the direct solver's band factor is valid for one
    int64_t k_version = 0;
    // direct solver (direct.cu): RCM rank of each particle, the band (factor) and its workspace
    int *band_rank = nullptr, *band_fail = nullptr;
    double *band_ab = nullptr, *band_y = nullptr;
    int64_t band_kd = 0, band_factored = -1;
    bool direct_off = false; // desc.direct == 2 and the band did not fit: the CG solves
    // fast assembly (assembly_fast.cu): per-bond T and Ts = T + T_opposite, per-particle U, the
    // 2-hop path lists (per slot counts, per row offsets, (partner bond, own bond) pairs) and the
    // flag of a bond broken in one direction only
    bool asm_fast = false;  // the path lists exist
    bool asm_exact = false; // lpmgpu_set_assembly_exact: the bit-exact kernel instead
    double *asm_T = nullptr, *asm_Ts = nullptr, *asm_U = nullptr;
    unsigned char *asm_cnt = nullptr, *asm_pa = nullptr;
    int64_t *asm_row = nullptr;
    int *asm_pb = nullptr, *asm_asym = nullptr;
    int64_t asm_paths = 0;
};

constexpr int kMaxGridBlocks = 4096;

// ---- kernels' host entry points (each enqueues on p.stream and returns a CUDA status)
cudaError_t build_topology(Problem &p, const double *xyz_host, int *err_code);
cudaError_t launch_geometry_force(Problem &p);
cudaError_t launch_update_rr(Problem &p);       // residual + norms into p.scal
cudaError_t launch_update_rr_impl(Problem &p, bool accumulate_reaction);
cudaError_t launch_k_to_f32(Problem &p);        // FP32 copy of K for the mixed-precision solve
// stiffness assembly with the BC elimination: the fast form (assembly_fast.cu) once its path
// lists exist and the handle is not in exact mode, else the bit-exact kernel (assembly.cu).
// With k32_written, the fast form also writes the FP32 copy and reports it there.
cudaError_t launch_assemble(Problem &p, bool apply_bc, bool *k32_written = nullptr);
cudaError_t launch_assemble_fast(Problem &p, bool apply_bc, bool write_k32);
cudaError_t setup_fast_assembly(Problem &p); // the 2-hop path lists, once per problem
// device-wide primitives of the set-up paths (prims.cu), enqueued on a stream
cudaError_t prim_exclusive_scan(cudaStream_t st, const int *in, int *out, int64_t count);
cudaError_t prim_exclusive_scan(cudaStream_t st, const int64_t *in, int64_t *out, int64_t count);
cudaError_t prim_max(cudaStream_t st, const int *in, int64_t count, int *dev_out);
// stable sort of (key, val) pairs by non-negative key
cudaError_t prim_sort_pairs(cudaStream_t st, const int *key, const int *val, int *skey, int *sval, int64_t n);
// each segment [off[s], off[s+1]) of non-negative values sorted ascending, in -> out
cudaError_t prim_segmented_sort(cudaStream_t st, const int *in, int *out, int64_t total, int nseg, const int *off);
cudaError_t launch_update_state_var(Problem &p);
cudaError_t launch_static_damage(Problem &p);   // sets p.scal->any_flag
// nonlocal damage (damage.cu): the neighbour search at creation, the averaged damage rate,
// and ParticleElasticDamage's state update
cudaError_t build_nonlocal(Problem &p, double cutoff_ratio);
cudaError_t build_nonlocal_lists(Problem &p, const int32_t *count, const int32_t *ids);
cudaError_t launch_nonlocal_average(Problem &p);
cudaError_t launch_edamage_update(Problem &p);
// fatigue (damage.cu): ParticleFatigueHCF's initial state variables and state update, and
// SolverFatigue::updateFatigueDamage (sets p.scal->any_flag)
cudaError_t launch_hcf_init(Problem &p);
cudaError_t launch_hcf_update(Problem &p);
cudaError_t launch_fatigue_damage(Problem &p, double dNdt);
cudaError_t launch_add_disp(Problem &p);        // xyz += x (solveLinearSystem position update)
cudaError_t launch_export_ref(const Problem &p, int64_t *IK, int64_t *JK, double *K); // device outputs
cudaError_t launch_apply_bc(Problem &p, const lpmgpu_load_step &s);

struct CGResult
{
    int64_t iters = 0;
    int64_t maxit_hits = 0;
    int refinements = 0;
    bool timeout = false;
    bool breakdown = false; // p.Ap == 0 in some launch
};
// Solves K x = res (current residual) into p.x with the reference's stopping rule.
cudaError_t solve_linear(Problem &p, CGResult &out);
// The same system by the band Cholesky (direct.cu); returns an LPMGPU status.
int32_t solve_direct(Problem &p);

// Pieces of the mixed-precision refinement, enqueued on p.stream without a host wait:
// r = res - K x with ||r||^2 copied to a pinned slot (read after the stream is synchronised),
// b32 = (float) r, and x += x32.
cudaError_t enqueue_true_residual(Problem &p);
double true_residual_result(const Problem &p);
cudaError_t enqueue_r_to_b32(Problem &p);
cudaError_t enqueue_res_to_b32(Problem &p); // b32 = (float) res: the first refinement, x = 0
cudaError_t enqueue_add_x32(Problem &p);

// Host-wait-free pieces of the load step (solver.cu), for callers that drive many problems:
// geometry + force state (+ updateRR) with the scalar record copied to p.scal_host; assembly
// (+ the FP32 copy in mixed precision); J2 state update + static damage with the scalar record;
// Assembly::storeStateVar / resetStateVar(true).
cudaError_t enqueue_force_state(Problem &p, bool with_rr);
cudaError_t enqueue_assemble(Problem &p, bool apply_bc);
cudaError_t enqueue_damage_update(Problem &p);
cudaError_t enqueue_store_state(Problem &p);
cudaError_t enqueue_reset_state(Problem &p);

// error text for lpmgpu_last_error
void set_last_error(const std::string &s);
// flushes and frees the handle's dump writer (waits for the steps it still writes)
void release_dump_writer(Problem &p);

template <typename T>
cudaError_t dalloc(Problem &p, T **ptr, size_t count)
{
    void *v = nullptr;
    size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMalloc(&v, bytes);
    if (e != cudaSuccess)
        return e;
    p.allocs.push_back(v);
    p.device_bytes += (int64_t)bytes;
    *ptr = static_cast<T *>(v);
    return cudaMemsetAsync(v, 0, bytes, p.stream);
}

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Bytes of matrix one CG iteration of the problem streams: its sliced-ELL block slots (nsb per
// lane of a 32-row slice), each d*d values in the CG's precision (FP32 for mixed) and a column.
inline int64_t cg_stream_bytes(const Problem &p)
{
    return p.nsb * kSlice * ((int64_t)p.dim * p.dim * (p.desc.precision == LPMGPU_MIXED ? 4 : 8) + 4);
}

} // namespace lpm

// the opaque handle of include/lpmgpu.h
struct lpmgpu_solver
{
    lpm::Problem p;
};
