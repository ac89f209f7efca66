// Nonlocal damage and the elastic-damage particle on the device:
//   Assembly::searchNonlocalNeighbors                  include/assembly.h:118-130
//   SolverStatic::updateStaticDamage (nonlocal rate)   include/solver_static.h:32-52, func_phi lpm.h:49-53
//   ParticleElasticDamage::updateParticleStateVariables include/particle_elastic_damage.h:159-170
//     with calcStrainEnergyDensity                     include/particle_elastic_damage.h:93-108
// The search keeps the reference's neighbour order (ascending id, the order of its inner loop),
// so the weighted sums of the averaging add in the reference's order.
#include <cub/cub.cuh>

#include "lpm_internal.cuh"

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

cudaError_t build_nonlocal(Problem &p, double cutoff_ratio)
{
    const int n = p.n;
    const double rc = cutoff_ratio * p.desc.nonlocal_L; // searchNonlocalNeighbors: cutoff_ratio * nonlocal_L
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
    size_t bytes = 0;
    if ((e = cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt, p.nlstart, n + 1, p.stream)) != cudaSuccess)
        return e;
    void *tmp = nullptr;
    if ((e = cudaMallocAsync(&tmp, bytes ? bytes : 16, p.stream)) != cudaSuccess)
        return e;
    e = cub::DeviceScan::ExclusiveSum(tmp, bytes, cnt, p.nlstart, n + 1, p.stream);
    cudaFreeAsync(tmp, p.stream);
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

} // namespace lpm
