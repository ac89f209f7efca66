// Host runtime of liblpmgpu: problem construction, the Newton loop, the damage loop and the
// load-step halving, and the C ABI of include/lpmgpu.h.  All heavy work is device kernels on
// the handle's stream; the host only reads back the few scalars each decision needs.
//   Solver::NewtonIteration           include/solver.h:55-90
//   SolverStatic::solveProblemStep    include/solver_static.h:99-152
//   SolverStatic::solveProblem        include/solver_static.h:65-96 (one load step per call)
//   Assembly::storeStateVar / resetStateVar  include/assembly.h:141-159
//   SolverFatigue::solveProblemStep / solveProblemStatic / solveProblemOneCycle /
//     updateFatigueDamage             include/solver_fatigue.h:76-302 (lpmgpu_fatigue_*)
// The force-state sequence of every Newton iteration and the state store / reset are captured
// into CUDA graphs when a problem is created and replayed (run_graph); the linear solve is the
// CG of cg.cu or, with desc.direct, the band Cholesky of direct.cu.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "lpm_internal.cuh"

namespace lpm
{

static thread_local std::string g_last_error;

void set_last_error(const std::string &s) { g_last_error = s; }

static int32_t cuda_fail(cudaError_t e, const char *what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation)
        return LPMGPU_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return LPMGPU_ERR_NO_DEVICE;
    return LPMGPU_ERR_CUDA;
}

#define CK(x)                                                                                                          \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return cuda_fail(e_, #x);                                                                                  \
    } while (0)

#define ST(x)                                                                                                          \
    do                                                                                                                 \
    {                                                                                                                  \
        int32_t s_ = (x);                                                                                              \
        if (s_ != LPMGPU_OK)                                                                                           \
            return s_;                                                                                                 \
    } while (0)

static int32_t sync_scalars(Problem &p)
{
    CK(cudaMemcpyAsync(p.scal_host, p.scal, sizeof(Scalars), cudaMemcpyDeviceToHost, p.stream));
    CK(cudaStreamSynchronize(p.stream));
    return LPMGPU_OK;
}

static cudaError_t enqueue_force_state_direct(Problem &p, bool with_rr)
{
    cudaError_t e = launch_geometry_force(p);
    if (e == cudaSuccess)
        e = launch_update_rr_impl(p, with_rr);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.scal_host, p.scal, sizeof(Scalars), cudaMemcpyDeviceToHost, p.stream);
    return e;
}

// A fixed sequence of the problem's work, captured into an executable graph at its first call and
// replayed afterwards.  The sequences given here read and write only the problem's own device
// buffers with constant arguments, so one capture serves every later call.  On any failure of the
// capture the problem goes back to direct launches for good.
template <typename F>
static void capture_graph(Problem &p, cudaGraphExec_t &slot, F enqueue_direct)
{
    if (!p.graphs_off && !slot)
    {
        const int64_t launches = p.ctr.kernel_launches;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess)
        {
            const cudaError_t e1 = enqueue_direct(p);
            e = cudaStreamEndCapture(p.stream, &graph);
            if (e == cudaSuccess)
                e = e1;
        }
        p.ctr.kernel_launches = launches;
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess && graph)
            e = cudaGraphInstantiate(&exec, graph, 0);
        if (graph)
            cudaGraphDestroy(graph);
        if (e != cudaSuccess || !exec)
        {
            p.graphs_off = true;
            (void)cudaGetLastError(); // the failed capture's error is not the caller's
        }
        else
            slot = exec;
    }
}

template <typename F>
static cudaError_t run_graph(Problem &p, cudaGraphExec_t &slot, int kernels, F enqueue_direct)
{
    capture_graph(p, slot, enqueue_direct);
    if (!p.graphs_off && slot)
    {
        const cudaError_t e = cudaGraphLaunch(slot, p.stream);
        if (e == cudaSuccess)
            p.ctr.kernel_launches += kernels;
        return e;
    }
    return enqueue_direct(p);
}

// Assembly::updateGeometry + updateForceState (and updateRR when with_rr), with the scalar record
// copied to p.scal_host: k_geometry_force, k_internal_force, k_finalize_rr and the copy
cudaError_t enqueue_force_state(Problem &p, bool with_rr)
{
    return run_graph(p, p.fs_graph[with_rr ? 1 : 0], 3,
                     [with_rr](Problem &q) { return enqueue_force_state_direct(q, with_rr); });
}

cudaError_t enqueue_assemble(Problem &p, bool apply_bc)
{
    p.k_version++;
    const bool mixed = p.desc.precision == LPMGPU_MIXED;
    bool k32 = false;
    cudaError_t e = launch_assemble(p, apply_bc, mixed ? &k32 : nullptr);
    if (e == cudaSuccess && mixed && !k32)
        e = launch_k_to_f32(p);
    return e;
}

cudaError_t enqueue_damage_update(Problem &p)
{
    cudaError_t e = launch_update_state_var(p);
    if (e == cudaSuccess)
        e = launch_static_damage(p);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.scal_host, p.scal, sizeof(Scalars), cudaMemcpyDeviceToHost, p.stream);
    return e;
}

// Assembly::updateGeometry + updateForceState (and updateRR when with_rr)
static int32_t force_state(Problem &p, bool with_rr)
{
    CK(cudaEventRecord(p.ev[0], p.stream));
    CK(enqueue_force_state(p, with_rr));
    CK(cudaEventRecord(p.ev[1], p.stream));
    CK(cudaStreamSynchronize(p.stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, p.ev[0], p.ev[1]);
    p.phase_s[0] += ms * 1e-3;
    p.ctr.force_seconds += ms * 1e-3;
    return LPMGPU_OK;
}

static int32_t assemble(Problem &p, bool apply_bc)
{
    CK(cudaEventRecord(p.ev[2], p.stream));
    CK(enqueue_assemble(p, apply_bc));
    CK(cudaEventRecord(p.ev[3], p.stream));
    CK(cudaEventSynchronize(p.ev[3]));
    float ms = 0;
    cudaEventElapsedTime(&ms, p.ev[2], p.ev[3]);
    p.phase_s[1] += ms * 1e-3;
    p.ctr.assembly_seconds += ms * 1e-3;
    return LPMGPU_OK;
}

// The direct solve in place of the CG (desc.direct 1), or after a CG that failed (desc.direct 2,
// while the band fits).  *used reports whether it ran.
static int32_t linear_solve_direct(Problem &p, lpmgpu_stats *st, bool *used)
{
    *used = false;
    if (!p.desc.direct || p.direct_off)
        return LPMGPU_OK;
    CK(cudaEventRecord(p.ev[4], p.stream));
    const int32_t r = solve_direct(p);
    if (r == LPMGPU_ERR_OUT_OF_MEMORY && p.desc.direct == 2 && !p.band_ab)
    {
        p.direct_off = true; // the band does not fit: the CG's result stands from now on
        return LPMGPU_OK;
    }
    ST(r);
    CK(cudaEventRecord(p.ev[5], p.stream));
    CK(cudaEventSynchronize(p.ev[5]));
    float ms = 0;
    cudaEventElapsedTime(&ms, p.ev[4], p.ev[5]);
    p.phase_s[2] += ms * 1e-3;
    *used = true;
    return LPMGPU_OK;
}

// One linear solve K x = res.  desc.direct 1: the band Cholesky.  desc.direct 2 (the drop-ins'
// SolverMode::PARDISO): the CG at the caller's tolerance first, and the band Cholesky only when
// the CG reached its cap or broke down.  Measured on B200 (hexagonal plates of 2,900 and 11,500
// particles, one factorisation and three solves per load step): the band solve took 20x and 58x
// the CG's time per load step, so the CG serves PARDISO mode and the factorisation is kept for
// the systems the CG cannot solve.
static int32_t linear_solve(Problem &p, lpmgpu_stats *st)
{
    bool direct = false;
    if (p.desc.direct == 1)
    {
        ST(linear_solve_direct(p, st, &direct));
        if (direct)
        {
            if (st)
            {
                st->newton_solves++;
                st->direct_solves++;
            }
            return LPMGPU_OK;
        }
    }
    CGResult r;
    CK(cudaEventRecord(p.ev[4], p.stream));
    CK(solve_linear(p, r));
    CK(cudaEventRecord(p.ev[5], p.stream));
    CK(cudaEventSynchronize(p.ev[5]));
    float ms = 0;
    cudaEventElapsedTime(&ms, p.ev[4], p.ev[5]);
    p.phase_s[2] += ms * 1e-3;
    if (r.timeout)
    {
        set_last_error("a device-side barrier wait timed out in the CG kernel");
        return LPMGPU_ERR_TIMEOUT;
    }
    if (p.desc.direct == 2 && (r.maxit_hits > 0 || r.breakdown))
        ST(linear_solve_direct(p, st, &direct));
    if (st)
    {
        st->newton_solves++;
        st->cg_iters += r.iters;
        st->cg_maxit_hits += r.maxit_hits;
        st->refinements += r.refinements;
        st->direct_solves += direct ? 1 : 0;
    }
    return LPMGPU_OK;
}

// Solver::NewtonIteration (solver.h:55-90): K fixed, positions += disp per iteration.
// *ni gets the iteration count, or max_iter on failure.
static int32_t newton(Problem &p, lpmgpu_stats *st, int *ni)
{
    ST(force_state(p, true));
    double nres = std::sqrt(p.scal_host->res_sq);
    const double nreac = std::sqrt(p.scal_host->reaction_sq);
    const double tol_mult = std_max(nres, nreac);
    int k = 0;
    while (nres > p.desc.tol_iter * tol_mult)
    {
        if (++k > p.desc.max_iter)
        {
            *ni = p.desc.max_iter;
            if (st)
                st->residual_norm = nres;
            return LPMGPU_OK;
        }
        if (p.desc.tangent)
            ST(assemble(p, true)); // tangent mode: K from the current state before every solve
        ST(linear_solve(p, st));
        CK(launch_add_disp(p));
        ST(force_state(p, true));
        nres = std::sqrt(p.scal_host->res_sq);
    }
    if (st)
        st->residual_norm = nres;
    *ni = k;
    return LPMGPU_OK;
}

static cudaError_t enqueue_store_state_direct(Problem &p)
{
    const size_t n = p.n, nb = (size_t)p.nbonds;
    cudaError_t e = cudaSuccess;
    const std::pair<void *, const void *> cp[] = {{p.xyz_last, p.xyz},   {p.damage_last, p.damage},
                                                  {p.sv_last, p.sv},     {p.dis_last, p.dis},
                                                  {p.bdamage_last, p.bdamage}, {p.bforce_last, p.bforce},
                                                  {p.dLp_last, p.dLp}};
    const size_t bytes[] = {sizeof(double) * 3 * n, sizeof(double) * n, sizeof(double) * p.nsv * n,
                            sizeof(double) * nb,    sizeof(double) * nb, sizeof(double) * nb, sizeof(double) * nb};
    for (int k = 0; k < 7 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(cp[k].first, cp[k].second, bytes[k], cudaMemcpyDeviceToDevice, p.stream);
    return e;
}

static cudaError_t enqueue_reset_state_direct(Problem &p)
{
    const size_t n = p.n, nb = (size_t)p.nbonds;
    cudaError_t e = cudaSuccess;
    const std::pair<void *, const void *> cp[] = {{p.xyz, p.xyz_last},   {p.damage, p.damage_last},
                                                  {p.sv, p.sv_last},     {p.dis, p.dis_last},
                                                  {p.bdamage, p.bdamage_last}, {p.bforce, p.bforce_last},
                                                  {p.dLp, p.dLp_last}};
    const size_t bytes[] = {sizeof(double) * 3 * n, sizeof(double) * n, sizeof(double) * p.nsv * n,
                            sizeof(double) * nb,    sizeof(double) * nb, sizeof(double) * nb, sizeof(double) * nb};
    for (int k = 0; k < 7 && e == cudaSuccess; ++k)
        e = cudaMemcpyAsync(cp[k].first, cp[k].second, bytes[k], cudaMemcpyDeviceToDevice, p.stream);
    return e;
}

cudaError_t enqueue_store_state(Problem &p)
{
    return run_graph(p, p.state_graph[0], 0, enqueue_store_state_direct);
}

cudaError_t enqueue_reset_state(Problem &p)
{
    return run_graph(p, p.state_graph[1], 0, enqueue_reset_state_direct);
}

// Captures every graph of the problem while nothing else uses its stream (at creation), so no
// capture later overlaps another thread's work on this problem (the dump writer's waits)
static void prepare_graphs(Problem &p)
{
    for (int rr = 0; rr < 2; ++rr)
        capture_graph(p, p.fs_graph[rr], [rr](Problem &q) { return enqueue_force_state_direct(q, rr != 0); });
    capture_graph(p, p.state_graph[0], enqueue_store_state_direct);
    capture_graph(p, p.state_graph[1], enqueue_reset_state_direct);
}

static int32_t store_state(Problem &p)
{
    CK(enqueue_store_state(p));
    return LPMGPU_OK;
}

static int32_t reset_state(Problem &p)
{
    CK(enqueue_reset_state(p));
    return LPMGPU_OK;
}

// SolverStatic::solveProblemStep: returns LPMGPU_OK or LPMGPU_ERR_NEWTON
static int32_t problem_step(Problem &p, const lpmgpu_load_step &s, lpmgpu_stats *st)
{
    CK(launch_apply_bc(p, s));
    int n_newton = 0;
    bool new_damaged = false;
    do
    {
        if (st)
            st->damage_iters++;
        if (!p.desc.tangent)
            ST(assemble(p, true));
        ST(newton(p, st, &n_newton));
        if (n_newton >= p.desc.max_iter)
            break;
        CK(launch_update_state_var(p));
        CK(launch_static_damage(p));
        ST(sync_scalars(p));
        new_damaged = p.scal_host->any_flag != 0;
        ST(store_state(p));
        if (new_damaged)
            ST(force_state(p, false));
    } while (new_damaged);
    if (st)
        st->reaction_norm = std::sqrt(p.scal_host->reaction_sq);
    return n_newton < p.desc.max_iter ? LPMGPU_OK : LPMGPU_ERR_NEWTON;
}

static int32_t scaled_step(Problem &p, const lpmgpu_load_step &s, double scale, lpmgpu_stats *st, int depth)
{
    std::vector<lpmgpu_dispbc> db(s.disp, s.disp + s.ndisp);
    std::vector<lpmgpu_forcebc> fb(s.force, s.force + s.nforce);
    for (auto &d : db)
        d.step *= scale;
    for (auto &f : fb)
    {
        f.fx *= scale;
        f.fy *= scale;
        f.fz *= scale;
    }
    lpmgpu_load_step sc{db.data(), s.ndisp, fb.data(), s.nforce};
    int32_t r = problem_step(p, sc, st);
    if (r != LPMGPU_ERR_NEWTON)
        return r;
    if (depth >= 30)
        return LPMGPU_ERR_CUTS;
    // solver_static.h:78-87: reset to the last converged state, halve, run both halves
    ST(reset_state(p));
    if (st)
        st->cuts++;
    ST(scaled_step(p, s, scale / 2.0, st, depth + 1));
    return scaled_step(p, s, scale / 2.0, st, depth + 1);
}

// SolverFatigue::solveProblemStep (solver_fatigue.h:278-302): BCs, K from the current state, Newton
static int32_t fatigue_step(Problem &p, const lpmgpu_load_step &s, lpmgpu_stats *st)
{
    CK(launch_apply_bc(p, s));
    if (!p.desc.tangent)
        ST(assemble(p, true));
    int n_newton = 0;
    ST(newton(p, st, &n_newton));
    if (st)
        st->reaction_norm = std::sqrt(p.scal_host->reaction_sq);
    return n_newton < p.desc.max_iter ? LPMGPU_OK : LPMGPU_ERR_NEWTON;
}

// one load step of SolverFatigue::solveProblemStatic (solver_fatigue.h:244-275): on failure reset
// to the last stored state, halve, run both halves; each converged (sub)step is followed by
// updateStateVar and storeStateVar
static int32_t fatigue_static_rec(Problem &p, const lpmgpu_load_step &s, double scale, lpmgpu_stats *st, int depth)
{
    std::vector<lpmgpu_dispbc> db(s.disp, s.disp + s.ndisp);
    std::vector<lpmgpu_forcebc> fb(s.force, s.force + s.nforce);
    for (auto &d : db)
        d.step *= scale;
    for (auto &f : fb)
    {
        f.fx *= scale;
        f.fy *= scale;
        f.fz *= scale;
    }
    lpmgpu_load_step sc{db.data(), s.ndisp, fb.data(), s.nforce};
    int32_t r = fatigue_step(p, sc, st);
    if (r == LPMGPU_OK)
    {
        CK(launch_update_state_var(p));
        ST(store_state(p));
        return LPMGPU_OK;
    }
    if (r != LPMGPU_ERR_NEWTON)
        return r;
    if (depth >= 30)
        return LPMGPU_ERR_CUTS;
    ST(reset_state(p));
    if (st)
        st->cuts++;
    ST(fatigue_static_rec(p, s, scale / 2.0, st, depth + 1));
    return fatigue_static_rec(p, s, scale / 2.0, st, depth + 1);
}

// SolverFatigue::updateFatigueDamage (solver_fatigue.h:76-126)
static int32_t fatigue_damage(Problem &p, double dNdt, int32_t *any)
{
    CK(launch_fatigue_damage(p, dNdt));
    ST(sync_scalars(p));
    if (any)
        *any = p.scal_host->any_flag != 0;
    return LPMGPU_OK;
}

// ---- lattice generators (include/utilities.h:93-310), host side
static void rmatrix(int f, const double a[3], double R[9])
{
    const double a1 = a[0], a2 = a[1], a3 = a[2];
    if (f == 0)
    {
        R[0] = cos(a2) * cos(a3);
        R[1] = -cos(a2) * sin(a3);
        R[2] = sin(a2);
        R[3] = cos(a1) * sin(a3) + sin(a1) * sin(a2) * cos(a3);
        R[4] = cos(a1) * cos(a3) - sin(a1) * sin(a2) * sin(a3);
        R[5] = -sin(a1) * cos(a2);
        R[6] = sin(a1) * sin(a3) - cos(a1) * sin(a2) * cos(a3);
        R[7] = sin(a1) * cos(a3) + cos(a1) * sin(a2) * sin(a3);
        R[8] = cos(a1) * cos(a2);
    }
    else if (f == 1)
    {
        R[0] = -cos(a1) * cos(a2) * cos(a3) - sin(a1) * sin(a3);
        R[1] = cos(a3) * sin(a1) - sin(a3) * cos(a2) * cos(a1);
        R[2] = sin(a2) * cos(a1);
        R[3] = sin(a3) * cos(a1) - cos(a3) * cos(a2) * sin(a1);
        R[4] = -cos(a1) * cos(a3) - sin(a1) * cos(a2) * sin(a3);
        R[5] = sin(a2) * sin(a1);
        R[6] = cos(a3) * sin(a2);
        R[7] = sin(a3) * sin(a2);
        R[8] = cos(a2);
    }
    else
    {
        R[0] = -sin(a1) * cos(a2) * sin(a3) + cos(a1) * cos(a3);
        R[1] = -sin(a3) * cos(a1) - cos(a3) * cos(a2) * sin(a1);
        R[2] = sin(a1) * sin(a2);
        R[3] = cos(a3) * sin(a1) + sin(a3) * cos(a2) * cos(a1);
        R[4] = -sin(a1) * sin(a3) + cos(a1) * cos(a2) * cos(a3);
        R[5] = -cos(a1) * sin(a2);
        R[6] = sin(a2) * sin(a3);
        R[7] = sin(a2) * cos(a3);
        R[8] = cos(a2);
    }
}

struct Gen
{
    double *out;
    int64_t cap, n = 0;
    const double *box;
    const double *R;
    bool check_z;
    void add(double x, double y, double z, bool z_from_rot = true)
    {
        const double p[3] = {x, y, z};
        double q[3];
        for (int i = 0; i < 3; ++i)
        {
            double s = 0.0;
            for (int j = 0; j < 3; ++j)
                s += R[3 * i + j] * p[j];
            q[i] = 1.0 * s;
        }
        if (!(q[0] >= box[0] && q[0] <= box[1] && q[1] >= box[2] && q[1] <= box[3]))
            return;
        if (check_z && !(q[2] >= box[4] && q[2] <= box[5]))
            return;
        if (out && n < cap)
        {
            out[3 * n] = q[0];
            out[3 * n + 1] = q[1];
            out[3 * n + 2] = z_from_rot ? q[2] : 0.0;
        }
        n++;
    }
};

static int64_t generate(int lattice, double r, const double *box, const double *R, double *out, int64_t cap)
{
    Gen g{out, cap, 0, box, R, lattice >= LPMGPU_SC3D};
    if (lattice == LPMGPU_SQUARE2D)
    {
        const double a = sqrt((box[1] - box[0]) * (box[1] - box[0]) + (box[3] - box[2]) * (box[3] - box[2]));
        const double hx = 2 * r, hy = hx;
        const int first = (int)floor((a - -a) / hx), rows = (int)floor((a - -a) / hy);
        for (int j = 1; j <= rows; j++)
            for (int i = 1; i <= first; i++)
                g.add(-a + hx * (i - 1) + r, -a + hy * (j - 1) + r, 0, false);
    }
    else if (lattice == LPMGPU_HEXAGON2D)
    {
        const double a = sqrt((box[1] - box[0]) * (box[1] - box[0]) + (box[3] - box[2]) * (box[3] - box[2]));
        const double hx = 2 * r, hy = hx * sqrt(3.0) / 2.0;
        const int first = 1 + (int)floor((a - -a) / hx), rows = 1 + (int)floor((a - -a) / hy);
        for (int j = 1; j <= rows; j++)
        {
            const double y = -a + hy * (j - 1);
            if (j % 2 == 1)
                for (int i = 1; i <= first; i++)
                    g.add(-a + hx * (i - 1), y, 0);
            else
                for (int i = 1; i <= first - 1; i++)
                    g.add(-a + hx * (2 * i - 1) / 2.0, y, 0);
        }
    }
    else if (lattice == LPMGPU_SC3D)
    {
        const double a = sqrt((box[1] - box[0]) * (box[1] - box[0]) + (box[3] - box[2]) * (box[3] - box[2]) +
                              (box[5] - box[4]) * (box[5] - box[4]));
        const double h = 2 * r;
        const int first = 1 + (int)floor((a - -a) / h), rows = first, layers = first;
        for (int k = 1; k <= layers; k++)
            for (int j = 1; j <= rows; j++)
                for (int i = 1; i <= first; i++)
                    g.add(box[0] + h * (i - 1), -a + h * (j - 1), -a + h * (k - 1));
    }
    else if (lattice == LPMGPU_FCC3D)
    {
        const double a = sqrt((box[1] - box[0]) * (box[1] - box[0]) + (box[3] - box[2]) * (box[3] - box[2]) +
                              (box[5] - box[4]) * (box[5] - box[4]));
        const double h = 4 * r / sqrt(2.0);
        const int first = 1 + (int)floor((a - -a) / h);
        const int rows = 1 + (int)floor((a - -a) / (h / 2.0)), layers = rows;
        for (int k = 1; k <= layers; k++)
        {
            const double z = -a + h / 2.0 * (k - 1);
            for (int j = 1; j <= rows; j++)
            {
                const double y = -a + h / 2.0 * (j - 1);
                const bool full = ((k % 2 == 1) == (j % 2 == 1));
                const int cnt = full ? first : first - 1;
                for (int i = 1; i <= cnt; i++)
                    g.add(full ? -a + h * (i - 1) : -a + h * (i - 1) + h / 2.0, y, z);
            }
        }
    }
    else
    {
        // BCC (no reference generator): cubic cell 4r/sqrt(3), corner and body-centre sites
        const double a = sqrt((box[1] - box[0]) * (box[1] - box[0]) + (box[3] - box[2]) * (box[3] - box[2]) +
                              (box[5] - box[4]) * (box[5] - box[4]));
        const double h = 4 * r / sqrt(3.0);
        const int first = 1 + (int)floor((a - -a) / h), layers = 1 + (int)floor((a - -a) / (h / 2.0));
        for (int k = 1; k <= layers; k++)
        {
            const double z = -a + h / 2.0 * (k - 1);
            const bool corner = (k % 2 == 1);
            const int cnt = corner ? first : first - 1;
            for (int j = 1; j <= cnt; j++)
                for (int i = 1; i <= cnt; i++)
                    g.add(corner ? -a + h * (i - 1) : -a + h * (i - 1) + h / 2.0,
                          corner ? -a + h * (j - 1) : -a + h * (j - 1) + h / 2.0, z);
        }
    }
    return g.n;
}

} // namespace lpm

using namespace lpm;

cudaError_t lpm::launch_update_rr(Problem &p) { return launch_update_rr_impl(p, true); }

extern "C" {

const char *lpmgpu_version(void) { return "lpmgpu 0.1 (sm_100a)"; }

const char *lpmgpu_status_string(int32_t s)
{
    switch (s)
    {
    case LPMGPU_OK: return "ok";
    case LPMGPU_ERR_INVALID_ARG: return "invalid argument";
    case LPMGPU_ERR_CUDA: return "CUDA error";
    case LPMGPU_ERR_OUT_OF_MEMORY: return "out of device memory";
    case LPMGPU_ERR_NEWTON: return "Newton iteration did not converge";
    case LPMGPU_ERR_CG_MAXIT: return "CG reached its iteration cap";
    case LPMGPU_ERR_TIMEOUT: return "device wait timed out";
    case LPMGPU_ERR_TOPOLOGY: return "unsupported particle topology";
    case LPMGPU_ERR_BUDGET: return "HBM budget exceeded";
    case LPMGPU_ERR_CUTS: return "load step halved too many times";
    case LPMGPU_ERR_NOT_READY: return "result not ready";
    case LPMGPU_ERR_NO_DEVICE: return "no CUDA device";
    case LPMGPU_ERR_NOT_SPD: return "stiffness not positive definite";
    case LPMGPU_ERR_CG_BREAKDOWN: return "CG broke down (p.Ap == 0)";
    default: return "unknown status";
    }
}

const char *lpmgpu_last_error(void) { return g_last_error.c_str(); }

int32_t lpmgpu_generate_lattice(int32_t lattice, double radius, const double box[6], int32_t euler_flag,
                                const double angles[3], double *out, int64_t cap, int64_t *count)
{
    if (!box || !angles || !count || lattice < 0 || lattice > LPMGPU_BCC3D || !(radius > 0))
        return LPMGPU_ERR_INVALID_ARG;
    double R[9];
    rmatrix(euler_flag, angles, R);
    *count = generate(lattice, radius, box, R, out, out ? cap : 0);
    return LPMGPU_OK;
}

static void free_problem(Problem &p)
{
    for (auto *slots : {p.fs_graph, p.state_graph})
        for (int k = 0; k < 2; ++k)
            if (slots[k])
            {
                cudaGraphExecDestroy(slots[k]);
                slots[k] = nullptr;
            }
    for (void *v : p.allocs)
        cudaFree(v);
    p.allocs.clear();
    if (p.scal_host)
        cudaFreeHost(p.scal_host);
    if (p.cg_info_host)
        cudaFreeHost(p.cg_info_host);
    for (auto &e : p.ev)
        if (e)
            cudaEventDestroy(e);
    for (auto &e : p.cg_ev)
        if (e)
            cudaEventDestroy(e);
    if (p.stream)
        cudaStreamDestroy(p.stream);
}

int32_t lpmgpu_create(const lpmgpu_desc *d, lpmgpu_solver **out)
{
    if (!d || !out || !d->xyz || d->n <= 0 || d->lattice < 0 || d->lattice > LPMGPU_BCC3D ||
        (d->ptype != LPMGPU_ELASTIC && d->ptype != LPMGPU_ELASTIC_DAMAGE && d->ptype != LPMGPU_J2 &&
         d->ptype != LPMGPU_FATIGUE_HCF) ||
        !(d->radius > 0) || d->max_iter < 0 || d->nonlocal_cutoff_ratio < 0 || d->direct < 0 || d->direct > 2)
        return LPMGPU_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    {
        set_last_error("no CUDA device visible; liblpmgpu has no CPU path");
        return LPMGPU_ERR_NO_DEVICE;
    }
    auto *h = new lpmgpu_solver();
    Problem &p = h->p;
    p.desc = *d;
    p.device = d->device;
    p.xyz0_host.assign(d->xyz, d->xyz + 3 * (size_t)d->n);
    if (d->type)
        p.type_host.assign(d->type, d->type + d->n);
    else
        p.type_host.assign(d->n, 0);
    for (auto &e : p.ev)
        e = nullptr;
    auto fail = [&](int32_t code) {
        free_problem(p);
        delete h;
        return code;
    };
#define CKF(x)                                                                                                         \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return fail(cuda_fail(e_, #x));                                                                            \
    } while (0)
    CKF(cudaSetDevice(p.device));
    CKF(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
    CKF(cudaDeviceGetAttribute(&p.num_sms, cudaDevAttrMultiProcessorCount, p.device));
    for (auto &e : p.ev)
        CKF(cudaEventCreate(&e));
    for (auto &e : p.cg_ev)
        CKF(cudaEventCreate(&e));
    p.graphs_off = std::getenv("LPMGPU_NO_GRAPHS") != nullptr;
    p.cell = make_cell(d->lattice, d->radius);
    p.n = d->n;
    p.dim = p.cell.dim;
    p.nsv = (d->ptype == LPMGPU_J2) ? 7 : (d->ptype == LPMGPU_FATIGUE_HCF) ? 3 : 1;
    if (d->C11 > 0 && d->ptype != LPMGPU_J2)
    {
        const double Ce[3] = {d->C11, d->C12, d->C44};
        kntv_cij(p.cell, Ce, p.kntv);
    }
    else
        kntv(p.cell, d->plane_stress, d->E, d->mu, p.kntv);
    const size_t n = p.n;
    CKF(cudaMallocHost(&p.scal_host, sizeof(Scalars)));
    CKF(cudaMallocHost(&p.cg_info_host, 8 * sizeof(int64_t)));
    CKF(dalloc(p, &p.scal, 1));
    CKF(dalloc(p, &p.partials, 2 * std::max<size_t>((size_t)kMaxGridBlocks, n / 64 + 1) + 16));
    CKF(dalloc(p, &p.barrier, 4));
    CKF(dalloc(p, &p.cg_info, 8));
    CKF(dalloc(p, &p.xyz, 3 * n));
    CKF(dalloc(p, &p.xyz_last, 3 * n));
    CKF(dalloc(p, &p.pin, 3 * n));
    CKF(dalloc(p, &p.pex, 3 * n));
    CKF(dalloc(p, &p.stress, 6 * n));
    CKF(dalloc(p, &p.damage, n));
    CKF(dalloc(p, &p.damage_last, n));
    CKF(dalloc(p, &p.damage_visual, n));
    CKF(dalloc(p, &p.ddot_local, n));
    CKF(dalloc(p, &p.sv, p.nsv * n));
    CKF(dalloc(p, &p.sv_last, p.nsv * n));
    if (d->ptype == LPMGPU_FATIGUE_HCF)
        CKF(launch_hcf_init(p));
    CKF(dalloc(p, &p.cons, 3 * n));
    CKF(dalloc(p, &p.type, n));
    CKF(dalloc(p, &p.dLe_total, 2 * n));
    CKF(dalloc(p, &p.TdLe_total, 2 * n));
    CKF(dalloc(p, &p.cs_sum, 6 * n));
    CKF(cudaMemcpyAsync(p.xyz, d->xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, p.stream));
    CKF(cudaMemcpyAsync(p.xyz_last, d->xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, p.stream));
    if (d->type)
        CKF(cudaMemcpyAsync(p.type, d->type, sizeof(int) * n, cudaMemcpyHostToDevice, p.stream));
    if ((d->bond_nb0 || d->bond_nb1 || d->bond_p2) && !(d->bond_nb0 && d->bond_nb1 && d->bond_p2))
        return fail(LPMGPU_ERR_INVALID_ARG);
    if ((d->bond_kn || d->bond_tv || d->bond_damage) && !d->bond_p2)
    {
        set_last_error("per-bond arrays need the bond lists they refer to (bond_nb0/bond_nb1/bond_p2)");
        return fail(LPMGPU_ERR_INVALID_ARG);
    }
    if ((d->nonlocal_count != nullptr) != (d->nonlocal_ids != nullptr) ||
        (d->nonlocal_count && d->nonlocal_cutoff_ratio > 0))
    {
        set_last_error("nonlocal lists need both nonlocal_count and nonlocal_ids, and no nonlocal_cutoff_ratio");
        return fail(LPMGPU_ERR_INVALID_ARG);
    }
    if (d->nonlocal_count)
    {
        int64_t total = 0;
        for (int i = 0; i < d->n; ++i)
        {
            if (d->nonlocal_count[i] < 0)
                return fail(LPMGPU_ERR_INVALID_ARG);
            total += d->nonlocal_count[i];
        }
        if (total >= ((int64_t)1 << 31))
        {
            set_last_error("more than 2^31 - 1 nonlocal neighbour pairs");
            return fail(LPMGPU_ERR_INVALID_ARG);
        }
        for (int64_t q = 0; q < total; ++q)
            if (d->nonlocal_ids[q] < 0 || d->nonlocal_ids[q] >= d->n)
                return fail(LPMGPU_ERR_INVALID_ARG);
    }
    int topo_err = 0;
    CKF(build_topology(p, d->xyz, &topo_err));
    if (d->nonlocal_cutoff_ratio > 0)
        CKF(build_nonlocal(p, d->nonlocal_cutoff_ratio));
    else if (d->nonlocal_count)
        CKF(build_nonlocal_lists(p, d->nonlocal_count, d->nonlocal_ids));
    CKF(cudaStreamSynchronize(p.stream));
    // the host pointers of the description are only read during creation
    p.desc.xyz = nullptr;
    p.desc.type = nullptr;
    p.desc.bond_nb0 = p.desc.bond_nb1 = p.desc.bond_p2 = nullptr;
    p.desc.bond_kn = p.desc.bond_tv = p.desc.bond_damage = nullptr;
    p.desc.nonlocal_count = p.desc.nonlocal_ids = nullptr;
    if (topo_err)
    {
        set_last_error("a particle has no bonds, or more bonds / connections than supported");
        return fail(topo_err);
    }
    const size_t ndof = n * p.dim;
    CKF(dalloc(p, &p.K, (size_t)p.nsb * p.dim * p.dim * kSlice));
    CKF(dalloc(p, &p.diag_raw, ndof));
    CKF(dalloc(p, &p.res, ndof));
    CKF(dalloc(p, &p.x, ndof));
    CKF(dalloc(p, &p.r, ndof));
    CKF(dalloc(p, &p.p0, ndof));
    CKF(dalloc(p, &p.p1, ndof));
    CKF(dalloc(p, &p.q, ndof));
    if (d->precision == LPMGPU_MIXED)
    {
        CKF(dalloc(p, &p.K32, (size_t)p.nsb * p.dim * p.dim * kSlice));
        CKF(dalloc(p, &p.x32, ndof));
        CKF(dalloc(p, &p.r32, ndof));
        CKF(dalloc(p, &p.pa32, ndof));
        CKF(dalloc(p, &p.pb32, ndof));
        CKF(dalloc(p, &p.q32, ndof));
        CKF(dalloc(p, &p.b32, ndof));
        CKF(dalloc(p, &p.r32b, ndof));
        CKF(dalloc(p, &p.w32b, ndof));
        CKF(dalloc(p, &p.s32b, ndof));
    }
    if (!std::getenv("LPMGPU_ASSEMBLY_EXACT"))
        CKF(setup_fast_assembly(p));
    // the examples run updateGeometry + updateForceState before constructing the solver
    CKF(launch_geometry_force(p));
    CKF(launch_update_rr_impl(p, false));
    CKF(cudaStreamSynchronize(p.stream));
    prepare_graphs(p);
#undef CKF
    *out = h;
    return LPMGPU_OK;
}

int32_t lpmgpu_destroy(lpmgpu_solver *h)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    cudaSetDevice(h->p.device);
    cudaStreamSynchronize(h->p.stream);
    release_dump_writer(h->p);
    free_problem(h->p);
    delete h;
    return LPMGPU_OK;
}

int32_t lpmgpu_get_sizes(const lpmgpu_solver *h, lpmgpu_sizes *o)
{
    if (!h || !o)
        return LPMGPU_ERR_INVALID_ARG;
    const Problem &p = h->p;
    o->n = p.n;
    o->dim = p.dim;
    o->nbonds = p.nbonds;
    o->nnzb = p.nnzb;
    o->nnz_upper = p.nnz_upper;
    o->max_bonds = p.max_bonds;
    o->max_conns = p.max_conns;
    o->device_bytes = p.device_bytes;
    return LPMGPU_OK;
}

int32_t lpmgpu_get_topology(const lpmgpu_solver *h, int32_t *nb0, int32_t *nb1, int32_t *bond_p2, int32_t *nconn,
                            int32_t *nlq, int32_t *conns)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    const Problem &p = h->p;
    const size_t n = p.n;
    std::vector<int> nb(n), n0(n), cst(n + 1);
    CK(cudaSetDevice(p.device));
    CK(cudaMemcpy(nb.data(), p.nb, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(n0.data(), p.nb0, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cst.data(), p.cstart, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i)
    {
        if (nb0)
            nb0[i] = n0[i];
        if (nb1)
            nb1[i] = nb[i] - n0[i];
        if (nconn)
            nconn[i] = cst[i + 1] - cst[i];
    }
    if (bond_p2)
        CK(cudaMemcpy(bond_p2, p.bp2, sizeof(int) * p.nbonds, cudaMemcpyDeviceToHost));
    if (nlq)
        CK(cudaMemcpy(nlq, p.nlq, sizeof(int) * n, cudaMemcpyDeviceToHost));
    if (conns)
        CK(cudaMemcpy(conns, p.conns, sizeof(int) * p.nnzb, cudaMemcpyDeviceToHost));
    return LPMGPU_OK;
}

int32_t lpmgpu_get_nonlocal(const lpmgpu_solver *h, int32_t *count, int32_t *ids, int64_t *total)
{
    if (!h || !total)
        return LPMGPU_ERR_INVALID_ARG;
    const Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    *total = p.nlist ? p.nnl : 0;
    if (!p.nlist)
        return LPMGPU_OK;
    if (count)
    {
        std::vector<int> start((size_t)p.n + 1);
        CK(cudaMemcpy(start.data(), p.nlstart, sizeof(int) * ((size_t)p.n + 1), cudaMemcpyDeviceToHost));
        for (int i = 0; i < p.n; ++i)
            count[i] = start[i + 1] - start[i];
    }
    if (ids && p.nnl > 0)
        CK(cudaMemcpy(ids, p.nlist, sizeof(int) * (size_t)p.nnl, cudaMemcpyDeviceToHost));
    return LPMGPU_OK;
}

int32_t lpmgpu_update_force_state(lpmgpu_solver *h)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->p.device));
    return force_state(h->p, false);
}

int32_t lpmgpu_update_state_var(lpmgpu_solver *h)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->p.device));
    CK(launch_update_state_var(h->p));
    CK(cudaStreamSynchronize(h->p.stream));
    return LPMGPU_OK;
}

int32_t lpmgpu_update_rr(lpmgpu_solver *h, double *norm)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    CK(launch_update_rr_impl(p, true));
    ST(sync_scalars(p));
    if (norm)
        *norm = std::sqrt(p.scal_host->res_sq);
    return LPMGPU_OK;
}

int32_t lpmgpu_assemble(lpmgpu_solver *h, int32_t apply_bc)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->p.device));
    return assemble(h->p, apply_bc != 0);
}

int32_t lpmgpu_export_ref_csr(const lpmgpu_solver *h, int64_t *K_pointer, int64_t *IK, int64_t *JK, double *K)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    const Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    const size_t n = p.n, nnz = (size_t)p.nnz_upper;
    if (K_pointer)
        CK(cudaMemcpy(K_pointer, p.kp_ref, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost));
    if (!IK && !JK && !K)
        return LPMGPU_OK;
    int64_t *dIK = nullptr, *dJK = nullptr;
    double *dK = nullptr;
    CK(cudaMalloc(&dIK, sizeof(int64_t) * (p.dim * n + 1)));
    CK(cudaMalloc(&dJK, sizeof(int64_t) * (nnz + 1)));
    CK(cudaMalloc(&dK, sizeof(double) * (nnz + 1)));
    cudaError_t e = launch_export_ref(p, dIK, dJK, dK);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(p.stream);
    if (e == cudaSuccess && IK)
        e = cudaMemcpy(IK, dIK, sizeof(int64_t) * (p.dim * n + 1), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && JK)
        e = cudaMemcpy(JK, dJK, sizeof(int64_t) * nnz, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && K)
        e = cudaMemcpy(K, dK, sizeof(double) * nnz, cudaMemcpyDeviceToHost);
    cudaFree(dIK);
    cudaFree(dJK);
    cudaFree(dK);
    CK(e);
    return LPMGPU_OK;
}

int32_t lpmgpu_solve_linear(lpmgpu_solver *h, double *disp, lpmgpu_stats *st)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    if (st)
        std::memset(st, 0, sizeof *st);
    ST(linear_solve(p, st));
    if (disp)
        CK(cudaMemcpy(disp, p.x, sizeof(double) * p.n * p.dim, cudaMemcpyDeviceToHost));
    return LPMGPU_OK;
}

int32_t lpmgpu_set_assembly_exact(lpmgpu_solver *h, int32_t exact)
{
    if (!h || (exact != 0 && exact != 1))
        return LPMGPU_ERR_INVALID_ARG;
    h->p.asm_exact = exact != 0;
    return LPMGPU_OK;
}

int32_t lpmgpu_solve_direct(lpmgpu_solver *h, double *disp, lpmgpu_stats *st)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    if (st)
        std::memset(st, 0, sizeof *st);
    CK(cudaEventRecord(p.ev[4], p.stream));
    ST(solve_direct(p));
    CK(cudaEventRecord(p.ev[5], p.stream));
    CK(cudaEventSynchronize(p.ev[5]));
    if (st)
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.ev[4], p.ev[5]);
        st->newton_solves = 1;
        st->direct_solves = 1;
        st->converged = 1;
        st->seconds = ms * 1e-3;
    }
    if (disp)
        CK(cudaMemcpy(disp, p.x, sizeof(double) * p.n * p.dim, cudaMemcpyDeviceToHost));
    return LPMGPU_OK;
}

static int32_t check_step(const Problem &p, const lpmgpu_load_step *s)
{
    if (!s || (s->ndisp > 0 && !s->disp) || (s->nforce > 0 && !s->force))
        return LPMGPU_ERR_INVALID_ARG;
    for (int q = 0; q < s->ndisp; ++q)
    {
        const auto &b = s->disp[q];
        if (b.count < 0 || (b.count > 0 && !b.ids) || b.flag < 0 || b.flag > 2)
            return LPMGPU_ERR_INVALID_ARG;
        for (int k = 0; k < b.count; ++k)
            if (b.ids[k] < 0 || b.ids[k] >= p.n)
                return LPMGPU_ERR_INVALID_ARG;
    }
    for (int q = 0; q < s->nforce; ++q)
    {
        const auto &b = s->force[q];
        if (b.count < 0 || (b.count > 0 && !b.ids))
            return LPMGPU_ERR_INVALID_ARG;
        for (int k = 0; k < b.count; ++k)
            if (b.ids[k] < 0 || b.ids[k] >= p.n)
                return LPMGPU_ERR_INVALID_ARG;
    }
    return LPMGPU_OK;
}

int32_t lpmgpu_apply_load_step(lpmgpu_solver *h, const lpmgpu_load_step *s)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    ST(check_step(h->p, s));
    CK(cudaSetDevice(h->p.device));
    CK(launch_apply_bc(h->p, *s));
    return LPMGPU_OK;
}

int32_t lpmgpu_solve_problem_step(lpmgpu_solver *h, const lpmgpu_load_step *s, lpmgpu_stats *st)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    ST(check_step(h->p, s));
    CK(cudaSetDevice(h->p.device));
    if (st)
        std::memset(st, 0, sizeof *st);
    int32_t r = problem_step(h->p, *s, st);
    if (st)
        st->converged = (r == LPMGPU_OK);
    return r;
}

int32_t lpmgpu_solve_load_step(lpmgpu_solver *h, const lpmgpu_load_step *s, lpmgpu_stats *st)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    ST(check_step(h->p, s));
    Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    lpmgpu_stats local;
    lpmgpu_stats *S = st ? st : &local;
    std::memset(S, 0, sizeof *S);
    for (double &t : p.phase_s)
        t = 0;
    CK(cudaEventRecord(p.ev[6], p.stream));
    int32_t r = scaled_step(p, *s, 1.0, S, 0);
    CK(cudaEventRecord(p.ev[7], p.stream));
    CK(cudaEventSynchronize(p.ev[7]));
    float ms = 0;
    cudaEventElapsedTime(&ms, p.ev[6], p.ev[7]);
    S->seconds = ms * 1e-3;
    S->converged = (r == LPMGPU_OK);
    S->reaction_norm = std::sqrt(p.scal_host->reaction_sq);
    return r;
}

static int32_t begin_call(lpmgpu_solver *h, lpmgpu_stats *st)
{
    if (st)
        *st = lpmgpu_stats{};
    for (double &t : h->p.phase_s)
        t = 0;
    CK(cudaSetDevice(h->p.device));
    return LPMGPU_OK;
}

int32_t lpmgpu_fatigue_solve_step(lpmgpu_solver *h, const lpmgpu_load_step *s, lpmgpu_stats *st)
{
    if (!h || !s)
        return LPMGPU_ERR_INVALID_ARG;
    ST(check_step(h->p, s));
    ST(begin_call(h, st));
    const int32_t r = fatigue_step(h->p, *s, st);
    if (st)
        st->converged = r == LPMGPU_OK;
    return r;
}

int32_t lpmgpu_fatigue_static_step(lpmgpu_solver *h, const lpmgpu_load_step *s, lpmgpu_stats *st)
{
    if (!h || !s)
        return LPMGPU_ERR_INVALID_ARG;
    ST(check_step(h->p, s));
    ST(begin_call(h, st));
    const int32_t r = fatigue_static_rec(h->p, *s, 1.0, st, 0);
    if (st)
    {
        st->converged = r == LPMGPU_OK;
        st->reaction_norm = std::sqrt(h->p.scal_host->reaction_sq);
    }
    return r;
}

int32_t lpmgpu_fatigue_update_damage(lpmgpu_solver *h, double dNdt, int32_t *any_damaged)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->p.device));
    return fatigue_damage(h->p, dNdt, any_damaged);
}

int32_t lpmgpu_fatigue_cycle(lpmgpu_solver *h, const lpmgpu_load_step *steps, int32_t nsteps, double dNdt,
                             lpmgpu_stats *st, int32_t *any_damaged)
{
    if (!h || nsteps < 0 || (nsteps > 0 && !steps))
        return LPMGPU_ERR_INVALID_ARG;
    for (int32_t k = 0; k < nsteps; ++k)
        ST(check_step(h->p, &steps[k]));
    ST(begin_call(h, st));
    Problem &p = h->p;
    bool all = true;
    for (int32_t k = 0; k < nsteps; ++k)
    {
        // solver_fatigue.h:227-236: the step's convergence is not acted on
        const int32_t r = fatigue_step(p, steps[k], st);
        if (r == LPMGPU_ERR_NEWTON)
        {
            all = false;
            if (st)
                st->cuts++;
        }
        else if (r != LPMGPU_OK)
            return r;
        CK(launch_update_state_var(p));
    }
    ST(fatigue_damage(p, dNdt, any_damaged));
    ST(store_state(p));
    ST(force_state(p, false));
    if (st)
    {
        st->converged = all;
        st->reaction_norm = std::sqrt(p.scal_host->reaction_sq);
    }
    return LPMGPU_OK;
}

int32_t lpmgpu_store_state(lpmgpu_solver *h)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->p.device));
    ST(store_state(h->p));
    CK(cudaStreamSynchronize(h->p.stream));
    return LPMGPU_OK;
}

int32_t lpmgpu_reset_state(lpmgpu_solver *h)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->p.device));
    ST(reset_state(h->p));
    CK(cudaStreamSynchronize(h->p.stream));
    return LPMGPU_OK;
}

int32_t lpmgpu_read_state(const lpmgpu_solver *h, double *xyz, double *pin, double *stress, double *damage,
                          double *damage_visual, double *state_var, double *bdamage)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    const Problem &p = h->p;
    const size_t n = p.n;
    CK(cudaSetDevice(p.device));
    CK(cudaStreamSynchronize(p.stream));
    if (xyz)
        CK(cudaMemcpy(xyz, p.xyz, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    if (pin)
        CK(cudaMemcpy(pin, p.pin, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    if (stress)
        CK(cudaMemcpy(stress, p.stress, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost));
    if (damage)
        CK(cudaMemcpy(damage, p.damage, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (damage_visual)
        CK(cudaMemcpy(damage_visual, p.damage_visual, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (state_var)
        CK(cudaMemcpy(state_var, p.sv, sizeof(double) * p.nsv * n, cudaMemcpyDeviceToHost));
    if (bdamage)
        CK(cudaMemcpy(bdamage, p.bdamage, sizeof(double) * p.nbonds, cudaMemcpyDeviceToHost));
    return LPMGPU_OK;
}

int32_t lpmgpu_read_residual(const lpmgpu_solver *h, double *res)
{
    if (!h || !res)
        return LPMGPU_ERR_INVALID_ARG;
    const Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    CK(cudaStreamSynchronize(p.stream));
    CK(cudaMemcpy(res, p.res, sizeof(double) * p.n * p.dim, cudaMemcpyDeviceToHost));
    return LPMGPU_OK;
}

int32_t lpmgpu_set_xyz(lpmgpu_solver *h, const double *xyz)
{
    if (!h || !xyz)
        return LPMGPU_ERR_INVALID_ARG;
    Problem &p = h->p;
    CK(cudaSetDevice(p.device));
    CK(cudaMemcpyAsync(p.xyz, xyz, sizeof(double) * 3 * p.n, cudaMemcpyHostToDevice, p.stream));
    CK(cudaStreamSynchronize(p.stream));
    return LPMGPU_OK;
}

int32_t lpmgpu_get_counters(const lpmgpu_solver *h, lpmgpu_counters *out)
{
    if (!h || !out)
        return LPMGPU_ERR_INVALID_ARG;
    *out = h->p.ctr;
    return LPMGPU_OK;
}

int32_t lpmgpu_get_stream(const lpmgpu_solver *h, void **stream)
{
    if (!h || !stream)
        return LPMGPU_ERR_INVALID_ARG;
    *stream = (void *)h->p.stream;
    return LPMGPU_OK;
}

int32_t lpmgpu_get_phase_times(const lpmgpu_solver *h, double *t4)
{
    if (!h || !t4)
        return LPMGPU_ERR_INVALID_ARG;
    for (int k = 0; k < 4; ++k)
        t4[k] = h->p.phase_s[k];
    return LPMGPU_OK;
}

} // extern "C"
