// Nonlocal damage, the elastic-damage and fatigue particles on the device:
//   Assembly::searchNonlocalNeighbors                  include/assembly.h:118-130
//   SolverStatic::updateStaticDamage (nonlocal rate)   include/solver_static.h:32-52, func_phi lpm.h:49-53
//   ParticleElasticDamage::updateParticleStateVariables include/particle_elastic_damage.h:159-170
//     with calcStrainEnergyDensity                     include/particle_elastic_damage.h:93-108
//   ParticleFatigueHCF::updateParticleStateVariables    include/particle_fatigue_hcf.h:128-145
//     with calcEqEnergy                                include/particle_fatigue_hcf.h:83-125
//   SolverFatigue::updateFatigueDamage                 include/solver_fatigue.h:76-126
//     with updateParticleFatigueDamage                 include/particle_fatigue_hcf.h:148-160
// The search keeps the reference's neighbour order (ascending id, the order of its inner loop),
// so the weighted sums of the averaging add in the reference's order.  It tests all pairs up to
// kNlAllPairsMax particles and bins them into cells above (nonlocal_grid.cuh), with the same
// distance test and each list sorted to ascending id; the caller may also hand over its own
// lists (build_nonlocal_lists).

#include <cstdlib>
#include <vector>

#include "lpm_internal.cuh"
#include "nonlocal_grid.cuh"

namespace lpm
{

// Particle::distanceTo (particle.h:277-280) from particle i to particle j, pow(x, 2) as x * x
__device__ __forceinline__ double dist_to(const double *__restrict__ xyz, int i, int j)
{
    const double dx = xyz[3 * i] - xyz[3 * j], dy = xyz[3 * i + 1] - xyz[3 * j + 1], dz = xyz[3 * i + 2] - xyz[3 * j + 2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// One warp per particle i: the particles j with distanceTo(j) < rc, in ascending j.  Pass 0
// counts (cnt[i]); pass 1 writes the list at start[i].
template <int PASS>
__global__ void k_nonlocal_search(int n, const double *__restrict__ xyz, double rc, int *__restrict__ cnt,
                                  const int *__restrict__ start, int *__restrict__ list)
{
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= n)
        return; // whole warps: blockDim is a multiple of 32
    int c = 0, o = PASS ? start[i] : 0;
    for (int j0 = 0; j0 < n; j0 += 32)
    {
        const int j = j0 + lane;
        const bool hit = j < n && dist_to(xyz, i, j) < rc;
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (PASS && hit)
            list[o + __popc(m & ((1u << lane) - 1u))] = j;
        o += __popc(m);
        c += __popc(m);
    }
    if (!PASS && lane == 0)
        cnt[i] = c;
}

// Cell-grid search: one thread per particle collects its neighbours from the cells around it
// (nonlocal_grid.cuh); pass 0 counts, pass 1 writes them unsorted at start[i].
template <int PASS>
__global__ void k_nonlocal_grid(int n, const double *__restrict__ xyz, double rc, const int *__restrict__ cxyz, int d0,
                                int d1, int d2, const int *__restrict__ cell_start, const int *__restrict__ cell_ids,
                                int *__restrict__ cnt, const int *__restrict__ start, int *__restrict__ list)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int dims[3] = {d0, d1, d2};
    if (PASS == 0)
        cnt[i] = nlgrid::candidates(i, xyz, rc, cxyz + 3 * (int64_t)i, dims, cell_start, cell_ids, nullptr);
    else
        nlgrid::candidates(i, xyz, rc, cxyz + 3 * (int64_t)i, dims, cell_start, cell_ids, list + start[i]);
}

// Above this many particles the search bins them into cells instead of testing all pairs
// (LPMGPU_NL_GRID=1 / =0 forces either).
constexpr int kNlAllPairsMax = 16384;

static bool use_grid(int n)
{
    const char *f = std::getenv("LPMGPU_NL_GRID");
    if (f && f[0] == '1')
        return true;
    if (f && f[0] == '0')
        return false;
    return n > kNlAllPairsMax;
}

// The cell-grid search: the same lists as the all-pairs search (the same distance test; each list
// sorted to ascending id by a segmented sort), in O(n x neighbours) instead of O(n^2).
static cudaError_t build_nonlocal_grid(Problem &p, double rc)
{
    const int n = p.n;
    int dims[3];
    std::vector<int> cxyz, cell_start, cell_ids;
    if (!nlgrid::bin(p.xyz0_host.data(), n, rc, int64_t(1) << 26, dims, cxyz, cell_start, cell_ids))
        return cudaErrorInvalidValue;
    int *d_cxyz = nullptr, *d_cs = nullptr, *d_ci = nullptr, *cnt = nullptr, *unsorted = nullptr;
    void *tmp = nullptr;
    cudaError_t e = dalloc(p, &p.nlstart, (size_t)n + 1);
    auto cleanup = [&]() {
        for (void *q : {(void *)d_cxyz, (void *)d_cs, (void *)d_ci, (void *)cnt, (void *)unsorted, tmp})
            if (q)
                cudaFreeAsync(q, p.stream);
    };
    if (e == cudaSuccess)
        e = cudaMallocAsync(&d_cxyz, sizeof(int) * cxyz.size(), p.stream);
    if (e == cudaSuccess)
        e = cudaMallocAsync(&d_cs, sizeof(int) * cell_start.size(), p.stream);
    if (e == cudaSuccess)
        e = cudaMallocAsync(&d_ci, sizeof(int) * cell_ids.size(), p.stream);
    if (e == cudaSuccess)
        e = cudaMallocAsync(&cnt, sizeof(int) * ((size_t)n + 1), p.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_cxyz, cxyz.data(), sizeof(int) * cxyz.size(), cudaMemcpyHostToDevice, p.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_cs, cell_start.data(), sizeof(int) * cell_start.size(), cudaMemcpyHostToDevice, p.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_ci, cell_ids.data(), sizeof(int) * cell_ids.size(), cudaMemcpyHostToDevice, p.stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), p.stream);
    if (e != cudaSuccess)
    {
        cleanup();
        return e;
    }
    k_nonlocal_grid<0><<<div_up(n, 128), 128, 0, p.stream>>>(n, p.xyz, rc, d_cxyz, dims[0], dims[1], dims[2], d_cs,
                                                             d_ci, cnt, nullptr, nullptr);
    p.ctr.kernel_launches++;
    e = prim_exclusive_scan(p.stream, cnt, p.nlstart, (int64_t)n + 1);
    int total = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&total, p.nlstart + n, sizeof(int), cudaMemcpyDeviceToHost, p.stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(p.stream); // also keeps the host bins alive through their copies
    if (e == cudaSuccess)
    {
        p.nnl = total;
        e = dalloc(p, &p.nlist, (size_t)total);
    }
    if (e == cudaSuccess)
        e = dalloc(p, &p.ddot_nonlocal, (size_t)n);
    if (e == cudaSuccess)
        e = cudaMallocAsync(&unsorted, sizeof(int) * ((size_t)total + 1), p.stream);
    if (e == cudaSuccess)
    {
        k_nonlocal_grid<1><<<div_up(n, 128), 128, 0, p.stream>>>(n, p.xyz, rc, d_cxyz, dims[0], dims[1], dims[2], d_cs,
                                                                 d_ci, nullptr, p.nlstart, unsorted);
        p.ctr.kernel_launches++;
        e = cudaGetLastError();
    }
    // each particle's list in ascending id, the order of the reference's loop
    if (e == cudaSuccess)
        e = prim_segmented_sort(p.stream, unsorted, p.nlist, total, n, p.nlstart);
    cleanup();
    return e;
}

cudaError_t build_nonlocal(Problem &p, double cutoff_ratio)
{
    const int n = p.n;
    const double rc = cutoff_ratio * p.desc.nonlocal_L; // searchNonlocalNeighbors: cutoff_ratio * nonlocal_L
    if (use_grid(n) && rc > 0)
        return build_nonlocal_grid(p, rc);
    cudaError_t e = dalloc(p, &p.nlstart, (size_t)n + 1);
    if (e != cudaSuccess)
        return e;
    int *cnt = nullptr;
    if ((e = cudaMallocAsync(&cnt, sizeof(int) * ((size_t)n + 1), p.stream)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), p.stream)) != cudaSuccess)
        return e;
    const int threads = 256, blocks = div_up((int64_t)n * 32, threads);
    k_nonlocal_search<0><<<blocks, threads, 0, p.stream>>>(n, p.xyz, rc, cnt, nullptr, nullptr);
    p.ctr.kernel_launches++;
    e = prim_exclusive_scan(p.stream, cnt, p.nlstart, (int64_t)n + 1);
    cudaFreeAsync(cnt, p.stream);
    if (e != cudaSuccess)
        return e;
    int total = 0;
    if ((e = cudaMemcpyAsync(&total, p.nlstart + n, sizeof(int), cudaMemcpyDeviceToHost, p.stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(p.stream)) != cudaSuccess)
        return e;
    p.nnl = total;
    if ((e = dalloc(p, &p.nlist, (size_t)total)) != cudaSuccess)
        return e;
    if ((e = dalloc(p, &p.ddot_nonlocal, (size_t)n)) != cudaSuccess)
        return e;
    k_nonlocal_search<1><<<blocks, threads, 0, p.stream>>>(n, p.xyz, rc, nullptr, p.nlstart, p.nlist);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// The caller's nonlocal lists (Particle::neighbors_nonlocal of an Assembly on which
// searchNonlocalNeighbors ran), already checked on the host: counts >= 0, ids in [0, n).
cudaError_t build_nonlocal_lists(Problem &p, const int32_t *count, const int32_t *ids)
{
    const int n = p.n;
    std::vector<int> start((size_t)n + 1, 0);
    for (int i = 0; i < n; ++i)
        start[i + 1] = start[i] + count[i];
    const int total = start[n];
    cudaError_t e = dalloc(p, &p.nlstart, (size_t)n + 1);
    if (e == cudaSuccess)
        e = dalloc(p, &p.nlist, (size_t)total);
    if (e == cudaSuccess)
        e = dalloc(p, &p.ddot_nonlocal, (size_t)n);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p.nlstart, start.data(), sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, p.stream);
    if (e == cudaSuccess && total > 0)
        e = cudaMemcpyAsync(p.nlist, ids, sizeof(int) * (size_t)total, cudaMemcpyHostToDevice, p.stream);
    p.nnl = total;
    // the host offsets must outlive the copies
    const cudaError_t s = cudaStreamSynchronize(p.stream);
    return e != cudaSuccess ? e : s;
}

// SolverStatic::updateStaticDamage, first loop (solver_static.h:35-52): the nonlocal damage rate
// of each damageable particle, the func_phi- and volume-weighted mean of its nonlocal neighbours'
// local rates, at the current positions
__global__ void k_nonlocal_average(int n, int undamaged, double L, double pvol, int nneighbors,
                                   const int *__restrict__ type, const int *__restrict__ nb,
                                   const int *__restrict__ nlstart, const int *__restrict__ nlist,
                                   const double *__restrict__ xyz, const double *__restrict__ ddot_local,
                                   double *__restrict__ ddot_nonlocal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || type[i] == undamaged)
        return;
    double A = 0, dn = 0;
    for (int q = nlstart[i]; q < nlstart[i + 1]; ++q)
    {
        const int j = nlist[q];
        if (type[j] == undamaged)
            continue;
        const double dis = dist_to(xyz, i, j);
        const double V_m = pvol * nb[j] / nneighbors;
        // func_phi (lpm.h:49-53): pow(1 / (1 + pow(x / L, 8)), 2), the outer square as t * t
        const double t = 1 / (1 + pow(dis / L, 8.0));
        const double phi = t * t;
        dn += ddot_local[j] * phi * V_m;
        A += phi * V_m;
    }
    ddot_nonlocal[i] = dn / A;
}

cudaError_t launch_nonlocal_average(Problem &p)
{
    if (!p.nlist)
        return cudaSuccess;
    k_nonlocal_average<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.desc.undamaged_type, p.desc.nonlocal_L,
                                                               p.cell.pvol, p.cell.nneighbors, p.type, p.nb,
                                                               p.nlstart, p.nlist, p.xyz, p.ddot_local,
                                                               p.ddot_nonlocal);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// ParticleElasticDamage::updateParticleStateVariables: state_var[0] = the strain energy density
// (spring energy of each bond plus the volumetric term of each layer, per modified volume), and
// the local damage rate (1 / k1) x its increase once it passed the damage surface k0 + k1 D
__global__ void k_edamage_update(int n, double pvol, int nneighbors, double k0, double k1,
                                 const int *__restrict__ bstart, const int *__restrict__ nb0,
                                 const int *__restrict__ nb, const double *__restrict__ Kn,
                                 const double *__restrict__ dLe, const double *__restrict__ dLe_total,
                                 const double *__restrict__ TdLe_total, const double *__restrict__ damage,
                                 const double *__restrict__ sv_last, double *__restrict__ sv,
                                 double *__restrict__ ddot_local)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double V_m = pvol * nb[i] / nneighbors;
    const int b0 = bstart[i], b1 = b0 + nb0[i], be = bstart[i + 1];
    double energy = 0;
    for (int L = 0; L < 2; ++L)
    {
        const int lo = L == 0 ? b0 : b1, hi = L == 0 ? b1 : be;
        for (int b = lo; b < hi; ++b)
            energy += 0.5 * (Kn[b] * dLe[b] * dLe[b]) / V_m;
        energy += 0.5 * TdLe_total[2 * i + L] * dLe_total[2 * i + L] / V_m;
    }
    sv[i] = energy;
    const double delta = energy - sv_last[i];
    const double f = energy - k1 * damage[i] - k0;
    ddot_local[i] = (f > 0 && delta > 0) ? (1 / k1) * delta : 0;
}

cudaError_t launch_edamage_update(Problem &p)
{
    k_edamage_update<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.cell.pvol, p.cell.nneighbors, p.desc.k0, p.desc.k1,
                                                             p.bstart, p.nb0, p.nb, p.Kn, p.dLe, p.dLe_total,
                                                             p.TdLe_total, p.damage, p.sv_last, p.sv, p.ddot_local);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// The strain energy density of particle i: each bond's spring energy, then the layer's
// volumetric term, per modified volume, layer by layer in bond order.  It is
// calcStrainEnergyDensity (particle_elastic_damage.h:93-108) and the energy_total that
// calcEqEnergy returns (particle_fatigue_hcf.h:98-123).
__device__ __forceinline__ double energy_density(int i, double pvol, int nneighbors, const int *__restrict__ bstart,
                                                 const int *__restrict__ nb0, const int *__restrict__ nb,
                                                 const double *__restrict__ Kn, const double *__restrict__ dLe,
                                                 const double *__restrict__ dLe_total,
                                                 const double *__restrict__ TdLe_total)
{
    const double V_m = pvol * nb[i] / nneighbors;
    const int b0 = bstart[i], b1 = b0 + nb0[i], be = bstart[i + 1];
    double energy = 0;
    for (int L = 0; L < 2; ++L)
    {
        const int lo = L == 0 ? b0 : b1, hi = L == 0 ? b1 : be;
        for (int b = lo; b < hi; ++b)
            energy += 0.5 * (Kn[b] * dLe[b] * dLe[b]) / V_m;
        energy += 0.5 * TdLe_total[2 * i + L] * dLe_total[2 * i + L] / V_m;
    }
    return energy;
}

// ParticleFatigueHCF state variables: [0] the largest energy so far, [1] / [2] the smallest /
// largest energy of the current cycle.  Initial value {0, INT_MAX, 0} (particle_fatigue_hcf.h:27-28).
constexpr double kHcfMinStart = 2147483647.0;

__global__ void k_hcf_init(int n, double *__restrict__ sv, double *__restrict__ sv_last)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    sv[3 * (int64_t)i] = sv_last[3 * (int64_t)i] = 0;
    sv[3 * (int64_t)i + 1] = sv_last[3 * (int64_t)i + 1] = kHcfMinStart;
    sv[3 * (int64_t)i + 2] = sv_last[3 * (int64_t)i + 2] = 0;
}

cudaError_t launch_hcf_init(Problem &p)
{
    k_hcf_init<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.sv, p.sv_last);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// ParticleFatigueHCF::updateParticleStateVariables: the cycle's smallest and largest energy,
// the largest so far, and the local damage rate A pow(largest so far, B) pow(range, d) when the
// cycle's energy range is positive.  std::min(a, b) is (b < a) ? b : a, std::max(a, b) is
// (a < b) ? b : a.
__global__ void k_hcf_update(int n, double pvol, int nneighbors, double fA, double fB, double fd,
                             const int *__restrict__ bstart, const int *__restrict__ nb0, const int *__restrict__ nb,
                             const double *__restrict__ Kn, const double *__restrict__ dLe,
                             const double *__restrict__ dLe_total, const double *__restrict__ TdLe_total,
                             double *__restrict__ sv, double *__restrict__ ddot_local)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double e = energy_density(i, pvol, nneighbors, bstart, nb0, nb, Kn, dLe, dLe_total, TdLe_total);
    double *s = sv + 3 * (int64_t)i;
    const double s1 = (s[1] < e) ? s[1] : e;
    const double s2 = (e < s[2]) ? s[2] : e;
    const double s0 = (s2 < s[0]) ? s[0] : s2;
    s[0] = s0;
    s[1] = s1;
    s[2] = s2;
    ddot_local[i] = (s2 - s1 > 0) ? fA * pow(s0, fB) * pow(s2 - s1, fd) : 0;
}

cudaError_t launch_hcf_update(Problem &p)
{
    k_hcf_update<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.cell.pvol, p.cell.nneighbors, p.desc.fatigue_A,
                                                         p.desc.fatigue_B, p.desc.fatigue_d, p.bstart, p.nb0, p.nb,
                                                         p.Kn, p.dLe, p.dLe_total, p.TdLe_total, p.sv, p.ddot_local);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// SolverFatigue::updateFatigueDamage, second loop, with
// ParticleFatigueHCF::updateParticleFatigueDamage: damage += nonlocal rate x dNdt, set to 1 at
// the threshold, the cycle's energy extremes cleared, and the flag raised when the damage moved
// by more than 1e-3 since the last stored state.  Without a nonlocal search the rate is 0/0, as
// in the reference.  Other particle types keep the base class's no-op.
__global__ void k_fatigue_damage(int n, int hcf, int undamaged, double threshold, double dNdt,
                                 const int *__restrict__ type, const double *__restrict__ ddot_nl,
                                 double *__restrict__ damage, const double *__restrict__ damage_last,
                                 double *__restrict__ sv, Scalars *scal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || type[i] == undamaged || !hcf)
        return;
    volatile double zero = 0.0;
    const double rate = ddot_nl ? ddot_nl[i] : zero / zero;
    double d = damage[i] + rate * dNdt;
    if (d >= threshold)
        d = 1;
    damage[i] = d;
    sv[3 * (int64_t)i + 1] = kHcfMinStart;
    sv[3 * (int64_t)i + 2] = 0;
    if (fabs(d - damage_last[i]) > 1e-3)
        atomicExch(&scal->any_flag, 1);
}

cudaError_t launch_fatigue_damage(Problem &p, double dNdt)
{
    cudaError_t e = cudaMemsetAsync(&p.scal->any_flag, 0, sizeof(int), p.stream);
    if (e != cudaSuccess)
        return e;
    if ((e = launch_nonlocal_average(p)) != cudaSuccess)
        return e;
    k_fatigue_damage<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.desc.ptype == LPMGPU_FATIGUE_HCF ? 1 : 0,
                                                             p.desc.undamaged_type, p.desc.damage_threshold, dNdt,
                                                             p.type, p.ddot_nonlocal, p.damage, p.damage_last, p.sv,
                                                             p.scal);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

} // namespace lpm
