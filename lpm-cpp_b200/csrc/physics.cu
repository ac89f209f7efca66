// Per-Newton-iteration particle physics on the device.  The bond and force passes work on tiles of
// particles (per-bond terms one thread per bond, per-particle sums one thread per particle in the
// reference's bond order); the state updates run one thread per particle.  Every sum follows the
// reference's list order, so it rounds exactly as the reference's does:
//   Particle::updateBondsGeometry / Bond::updatebGeometry  include/particle.h:164-181, bond.h:30-39
//   ParticleElastic::updateBondsForce                      include/particle_elastic.h:38-50
//   ParticleJ2Plasticity::updateBondsForce                 include/particle_j2plasticity.h:63-76
//   ParticleElasticDamage::updateBondsForce                include/particle_elastic_damage.h:80-91
//   Particle::updateParticleForce / Stress / DamageVisual  include/particle.h:151-240
//   Solver::updateRR                                       include/solver.h:112-126
//   ParticleJ2Plasticity::updateParticleStateVariables     include/particle_j2plasticity.h:78-140
//   SolverStatic::updateStaticDamage                       include/solver_static.h:32-62
//   Solver::updateForceBC / updateDisplacementBC           include/solver.h:129-188
// The reference finds the opposite bond with a linear find_if per bond (particle.h:207);
// here it is the precomputed brev index.
#include "lpm_internal.cuh"

namespace lpm
{

struct PhysArgs
{
    int n, dim, ptype;
    const int *__restrict__ bstart, *__restrict__ nb0, *__restrict__ bp2, *__restrict__ brev;
    double *__restrict__ xyz;
    const double *__restrict__ dis0, *__restrict__ Kn, *__restrict__ Tv;
    double *__restrict__ dis, *__restrict__ dLe, *__restrict__ dLp, *__restrict__ bstrain, *__restrict__ cs;
    double *__restrict__ bforce, *__restrict__ bdamage;
    double *__restrict__ dLe_total, *__restrict__ TdLe_total, *__restrict__ cs_sum;
    const double *__restrict__ damage;
};

// Both per-Newton-iteration kernels work on tiles of kTileParticles consecutive particles,
// whose bonds are one contiguous range of the bond arrays.  Phase 1 runs one thread per BOND
// (every lane busy, every per-bond array read and written contiguously; only the partner's
// coordinates, damage and opposite bond are gathers) and leaves the per-bond terms of the
// particle sums in shared memory.  Phase 2 runs one thread per particle and adds its bonds'
// terms in bond order, the order of the reference's loops, so every sum rounds exactly as the
// reference's does.  Blocks loop over tiles, so the grid (and the per-block partials of the
// residual norms) stay bounded.
constexpr int kTileParticles = 32;
constexpr int kTileThreads = 256;

// owner (tile-local particle) of bond b, given the tile's bstart[p0 .. p0 + np] in shared memory
__device__ __forceinline__ int tile_owner(const int *bs, int np, int b)
{
    int lo = 0, hi = np - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (bs[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// updateBondsGeometry + updateBondsForce (particle.h:164-181, bond.h:30-39, particle_elastic.h:38-50)
__global__ void __launch_bounds__(kTileThreads) k_geometry_force(PhysArgs a, int maxb)
{
    extern __shared__ __align__(16) double tsm[];
    // per tile bond (<= kTileParticles * maxb): dLe, Tv dLe, cs[3]; per particle: the layer sums
    const int cap = kTileParticles * maxb;
    double *t_dle = tsm, *t_tdle = t_dle + cap, *t_c = t_tdle + cap, *t_dlt = t_c + 3 * cap;
    int *bs = reinterpret_cast<int *>(t_dlt + 2 * kTileParticles), *b1s = bs + kTileParticles + 1;
    const bool dmg_max = a.ptype == LPMGPU_J2 || a.ptype == LPMGPU_ELASTIC_DAMAGE || a.ptype == LPMGPU_FATIGUE_HCF;
    const int ntiles = (a.n + kTileParticles - 1) / kTileParticles;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int p0 = tile * kTileParticles, np = min(kTileParticles, a.n - p0);
        for (int q = threadIdx.x; q <= np; q += blockDim.x)
            bs[q] = a.bstart[p0 + q];
        for (int q = threadIdx.x; q < np; q += blockDim.x)
            b1s[q] = a.bstart[p0 + q] + a.nb0[p0 + q];
        __syncthreads();
        const int bb = bs[0], be = bs[np];
        // phase 1: one thread per bond
        for (int b = bb + threadIdx.x; b < be; b += blockDim.x)
        {
            const int o = tile_owner(bs, np, b), i = p0 + o;
            const int j = a.bp2[b];
            const double dx = a.xyz[3 * i] - a.xyz[3 * j], dy = a.xyz[3 * i + 1] - a.xyz[3 * j + 1],
                         dz = a.xyz[3 * i + 2] - a.xyz[3 * j + 2];
            const bool broken = fabs(a.bdamage[b] - 1.0) < kEps;
            const double dis = sqrt(dx * dx + dy * dy + dz * dz);
            const double d0 = a.dis0[b];
            const double dL = broken ? 0.0 : (dis - d0);
            const double bst = broken ? 0.0 : (dL / dis);
            const double dle = broken ? 0.0 : (dis - d0 - a.dLp[b]);
            const double c0 = broken ? 0.0 : (dx / dis);
            const double c1 = broken ? 0.0 : (dy / dis);
            const double c2 = broken ? 0.0 : (dz / dis);
            a.dis[b] = dis;
            a.bstrain[b] = bst;
            a.dLe[b] = dle;
            a.cs[3 * (int64_t)b] = c0;
            a.cs[3 * (int64_t)b + 1] = c1;
            a.cs[3 * (int64_t)b + 2] = c2;
            const int t = b - bb;
            t_dle[t] = dle;
            t_tdle[t] = a.Tv[b] * dle;
            t_c[3 * t] = c0;
            t_c[3 * t + 1] = c1;
            t_c[3 * t + 2] = c2;
        }
        __syncthreads();
        // phase 2: one thread per particle, each layer's sums in bond order
        if (threadIdx.x < np)
        {
            const int o = threadIdx.x, i = p0 + o;
            for (int L = 0; L < 2; ++L)
            {
                const int lo = (L == 0 ? bs[o] : b1s[o]) - bb, hi = (L == 0 ? b1s[o] : bs[o + 1]) - bb;
                double sd = 0, ts = 0, cx = 0, cy = 0, cz = 0;
                for (int t = lo; t < hi; ++t)
                {
                    sd += t_dle[t];
                    ts += t_tdle[t];
                    cx += t_c[3 * t];
                    cy += t_c[3 * t + 1];
                    cz += t_c[3 * t + 2];
                }
                t_dlt[2 * o + L] = sd;
                a.dLe_total[2 * i + L] = sd;
                a.TdLe_total[2 * i + L] = ts;
                a.cs_sum[6 * i + 3 * L] = cx;
                a.cs_sum[6 * i + 3 * L + 1] = cy;
                a.cs_sum[6 * i + 3 * L + 2] = cz;
            }
        }
        __syncthreads();
        // phase 3: one thread per bond, the bond force
        for (int b = bb + threadIdx.x; b < be; b += blockDim.x)
        {
            const int o = tile_owner(bs, np, b), i = p0 + o;
            const int L = b < b1s[o] ? 0 : 1;
            double f = 2. * a.Kn[b] * t_dle[b - bb] + 2. * a.Tv[b] * t_dlt[2 * o + L];
            double D = a.bdamage[b];
            if (dmg_max)
            {
                D = std_max(D, std_max(a.damage[i], a.damage[a.bp2[b]]));
                a.bdamage[b] = D;
            }
            f *= (1.0 - D);
            a.bforce[b] = f;
        }
        __syncthreads();
    }
}

struct ForceArgs
{
    int n, dim, nneighbors;
    double pvol;
    const int *__restrict__ bstart, *__restrict__ brev, *__restrict__ nb, *__restrict__ cons;
    const double *__restrict__ cs, *__restrict__ dis, *__restrict__ bforce, *__restrict__ bdamage,
        *__restrict__ pex;
    double *__restrict__ pin, *__restrict__ stress, *__restrict__ damage_visual, *__restrict__ res;
    double *__restrict__ partials; // [grid][2]: residual^2, reaction^2
};

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// deterministic block sum (fixed tree), result valid in thread 0
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        sh[w] = v;
    __syncthreads();
    double r = 0;
    if (w == 0)
    {
        r = (l < NT / 32) ? sh[l] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// updateParticleForce + updateParticleStress + updateParticleDamageVisual, then updateRR
// (particle.h:151-240, solver.h:112-126), in the tiles of k_geometry_force.  The per-block
// partials of the residual and reaction norms add each tile's particles in order and the tiles
// in order, so every run rounds alike.
__global__ void __launch_bounds__(kTileThreads) k_internal_force(ForceArgs a, int maxb)
{
    extern __shared__ __align__(16) double tsm[];
    __shared__ double sh[2 * kTileParticles];
    // per tile bond: the three Pin terms, the six stress terms and the bond damage
    const int cap = kTileParticles * maxb;
    double *t_v = tsm;
    int *bs = reinterpret_cast<int *>(t_v + 10 * cap);
    double rsq_blk = 0.0, rea_blk = 0.0; // valid in thread 0
    const int ntiles = (a.n + kTileParticles - 1) / kTileParticles;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int p0 = tile * kTileParticles, np = min(kTileParticles, a.n - p0);
        for (int q = threadIdx.x; q <= np; q += blockDim.x)
            bs[q] = a.bstart[p0 + q];
        __syncthreads();
        const int bb = bs[0], be = bs[np];
        for (int b = bb + threadIdx.x; b < be; b += blockDim.x)
        {
            const int o = tile_owner(bs, np, b), i = p0 + o;
            const double V_m = a.pvol * a.nb[i] / a.nneighbors;
            const double fs = a.bforce[b] + a.bforce[a.brev[b]];
            const double cx = a.cs[3 * (int64_t)b], cy = a.cs[3 * (int64_t)b + 1], cz = a.cs[3 * (int64_t)b + 2];
            const double w = 0.5 / V_m * (a.dis[b]) * 0.5 * fs;
            double *v = t_v + 10 * (b - bb);
            v[0] = cx * 0.5 * fs;
            v[1] = cy * 0.5 * fs;
            v[2] = cz * 0.5 * fs;
            v[3] = w * (cx) * (cx);
            v[4] = w * (cy) * (cy);
            v[5] = w * (cz) * (cz);
            v[6] = w * (cy) * (cz);
            v[7] = w * (cx) * (cz);
            v[8] = w * (cx) * (cy);
            v[9] = a.bdamage[b];
        }
        __syncthreads();
        double rsq = 0.0, rea = 0.0;
        if (threadIdx.x < np)
        {
            const int o = threadIdx.x, i = p0 + o;
            double P0 = 0., P1 = 0., P2 = 0.;
            double S0 = 0, S1 = 0, S2 = 0, S3 = 0, S4 = 0, S5 = 0, dv = 0;
            for (int t = bs[o] - bb; t < bs[o + 1] - bb; ++t)
            {
                const double *v = t_v + 10 * t;
                P0 += v[0];
                P1 += v[1];
                P2 += v[2];
                S0 += v[3];
                S1 += v[4];
                S2 += v[5];
                S3 += v[6];
                S4 += v[7];
                S5 += v[8];
                dv += v[9];
            }
            a.pin[3 * i] = P0;
            a.pin[3 * i + 1] = P1;
            a.pin[3 * i + 2] = P2;
            double *st = a.stress + 6 * (int64_t)i;
            st[0] = S0;
            st[1] = S1;
            st[2] = S2;
            st[3] = S3;
            st[4] = S4;
            st[5] = S5;
            const int nbi = a.nb[i];
            a.damage_visual[i] = dv / (double)nbi;
            const double P[3] = {P0, P1, P2};
            for (int k = 0; k < a.dim; ++k)
            {
                const int c = a.cons[3 * i + k];
                const double rv = (1 - c) * (a.pex[3 * i + k] - P[k]);
                a.res[(int64_t)a.dim * i + k] = rv;
                rsq += rv * rv;
                if (c == 1)
                    rea += P[k] * P[k];
            }
        }
        if (threadIdx.x < kTileParticles)
        {
            sh[threadIdx.x] = rsq;
            sh[kTileParticles + threadIdx.x] = rea;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < np; ++k)
            {
                rsq_blk += sh[k];
                rea_blk += sh[kTileParticles + k];
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        a.partials[2 * blockIdx.x] = rsq_blk;
        a.partials[2 * blockIdx.x + 1] = rea_blk;
    }
}

// fixed-order sum of the per-block partials; accumulates the reaction history
__global__ void k_finalize_rr(int nblk, const double *__restrict__ partials, Scalars *scal, int accumulate)
{
    __shared__ double sh[32];
    double r = 0, q = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    {
        r += partials[2 * b];
        q += partials[2 * b + 1];
    }
    const double R = block_sum<256>(r, sh);
    const double Q = block_sum<256>(q, sh);
    if (threadIdx.x == 0)
    {
        scal->res_sq = R;
        if (accumulate)
            scal->reaction_sq += Q;
    }
}

// grid of the tiled kernels: one block per tile up to 8 blocks per SM, then blocks loop over
// tiles (the per-block partials fit the 2 x kMaxGridBlocks buffer)
static int phys_grid(const Problem &p)
{
    const int64_t ntiles = (p.n + kTileParticles - 1) / kTileParticles;
    const int64_t cap = std::min<int64_t>((int64_t)p.num_sms * 8, kMaxGridBlocks);
    return (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, cap));
}

static size_t geo_smem(const Problem &p)
{
    return sizeof(double) * (5 * (size_t)kTileParticles * p.max_bonds + 2 * kTileParticles) +
           sizeof(int) * (2 * kTileParticles + 1);
}

static size_t force_smem(const Problem &p)
{
    return sizeof(double) * 10 * (size_t)kTileParticles * p.max_bonds + sizeof(int) * (kTileParticles + 1);
}

cudaError_t launch_geometry_force(Problem &p)
{
    PhysArgs a;
    a.n = p.n;
    a.dim = p.dim;
    a.ptype = p.desc.ptype;
    a.bstart = p.bstart;
    a.nb0 = p.nb0;
    a.bp2 = p.bp2;
    a.brev = p.brev;
    a.xyz = p.xyz;
    a.dis0 = p.dis0;
    a.Kn = p.Kn;
    a.Tv = p.Tv;
    a.dis = p.dis;
    a.dLe = p.dLe;
    a.dLp = p.dLp;
    a.bstrain = p.bstrain;
    a.cs = p.cs;
    a.bforce = p.bforce;
    a.bdamage = p.bdamage;
    a.dLe_total = p.dLe_total;
    a.TdLe_total = p.TdLe_total;
    a.cs_sum = p.cs_sum;
    a.damage = p.damage;
    const size_t smem = geo_smem(p);
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(k_geometry_force, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess)
            return e;
    }
    k_geometry_force<<<phys_grid(p), kTileThreads, smem, p.stream>>>(a, p.max_bonds);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// accumulate_reaction: Solver::updateRR appends the reaction forces to the history
// (solver.h:122-123); Assembly::updateForceState alone (solver_static.h:132-133) does not
cudaError_t launch_update_rr_impl(Problem &p, bool accumulate_reaction)
{
    ForceArgs a;
    a.n = p.n;
    a.dim = p.dim;
    a.nneighbors = p.cell.nneighbors;
    a.pvol = p.cell.pvol;
    a.bstart = p.bstart;
    a.brev = p.brev;
    a.nb = p.nb;
    a.cons = p.cons;
    a.cs = p.cs;
    a.dis = p.dis;
    a.bforce = p.bforce;
    a.bdamage = p.bdamage;
    a.pex = p.pex;
    a.pin = p.pin;
    a.stress = p.stress;
    a.damage_visual = p.damage_visual;
    a.res = p.res;
    a.partials = p.partials;
    const int nblk = phys_grid(p);
    const size_t smem = force_smem(p);
    if (smem > 48 * 1024)
    {
        const cudaError_t e = cudaFuncSetAttribute(k_internal_force, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess)
            return e;
    }
    k_internal_force<<<nblk, kTileThreads, smem, p.stream>>>(a, p.max_bonds);
    k_finalize_rr<<<1, 256, 0, p.stream>>>(nblk, p.partials, p.scal, accumulate_reaction ? 1 : 0);
    p.ctr.kernel_launches += 2;
    return cudaGetLastError();
}

// ParticleJ2Plasticity::updateParticleStateVariables (particle_j2plasticity.h:78-140)
__global__ void k_j2_update(int n, double E, double mu, double sigmay, double xi, double H, double A,
                            const int *__restrict__ bstart, const double *__restrict__ stress,
                            const double *__restrict__ dis, const double *__restrict__ cs, double *__restrict__ sv,
                            double *__restrict__ dLp, double *__restrict__ ddot_local)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double *s = sv + 7 * (int64_t)i;
    double st[6], dpl[6] = {0, 0, 0, 0, 0, 0};
    double sigma_eq = 0.0, triax = 0.0, dlambda = 0.0;
    for (int j = 0; j < 6; ++j)
        st[j] = stress[6 * (int64_t)i + j];
    const double sigma_m = 1.0 / 3.0 * (st[0] + st[1] + st[2]);
    for (int j = 0; j < 3; j++)
        st[j] -= sigma_m;
    for (int j = 0; j < 6; j++)
        st[j] -= s[j + 1];
    for (int j = 0; j < 6; j++)
    {
        if (j < 3)
            sigma_eq += st[j] * st[j];
        else
            sigma_eq += 2.0 * st[j] * st[j];
    }
    sigma_eq = sqrt(3.0 / 2.0 * sigma_eq);
    const double yield = sigma_eq - (sigmay + (1.0 - xi) * H * s[0]);
    const double G = E / 2 / (1 + mu);
    if (yield > 0.0)
        dlambda = yield / (3 * G + H);
    s[0] += dlambda;
    for (int j = 0; j < 6; j++)
        if (fabs(sigma_eq) > kEps)
        {
            dpl[j] = dlambda * 1.5 * st[j] / sigma_eq;
            s[j + 1] += 2. / 3. * xi * H * dpl[j];
        }
    for (int b = bstart[i]; b < bstart[i + 1]; ++b)
    {
        const double cx = cs[3 * (int64_t)b], cy = cs[3 * (int64_t)b + 1], cz = cs[3 * (int64_t)b + 2];
        const double ddLp = dis[b] * (dpl[0] * cx * cx + dpl[1] * cy * cy + dpl[2] * cz * cz + 2 * dpl[3] * cy * cz +
                                      2 * dpl[4] * cx * cz + 2 * dpl[5] * cx * cy);
        dLp[b] += ddLp;
    }
    if (sigma_eq > kEps)
        triax = sigma_m / sigma_eq;
    ddot_local[i] = dlambda * (1.0 + A * triax);
}

cudaError_t launch_update_state_var(Problem &p)
{
    if (p.desc.ptype == LPMGPU_ELASTIC_DAMAGE)
        return launch_edamage_update(p);
    if (p.desc.ptype == LPMGPU_FATIGUE_HCF)
        return launch_hcf_update(p);
    if (p.desc.ptype != LPMGPU_J2)
        return cudaSuccess;
    k_j2_update<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.desc.E, p.desc.mu, p.desc.sigmay, p.desc.xi, p.desc.H,
                                                        p.desc.A, p.bstart, p.stress, p.dis, p.cs, p.sv, p.dLp,
                                                        p.ddot_local);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// SolverStatic::updateStaticDamage.  The nonlocal rate comes from k_nonlocal_average when a
// nonlocal search ran; without one it is 0/0 (solver_static.h:39-51), exactly as in the reference
// when searchNonlocalNeighbors was not called.  Elastic particles ignore it; J2 and elastic-damage
// particles add it to their damage and set the damage to 1 at their threshold
// (particle_j2plasticity.h:142-152, particle_elastic_damage.h:172-181).
__global__ void k_static_damage(int n, int ptype, int undamaged, double critical, double threshold,
                                const int *__restrict__ type, const int *__restrict__ bstart,
                                const double *__restrict__ bstrain, const double *__restrict__ ddot_nl,
                                double *__restrict__ bdamage, double *__restrict__ damage,
                                const double *__restrict__ damage_last, Scalars *scal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || type[i] == undamaged)
        return;
    bool changed = false;
    if (ptype == LPMGPU_J2 || ptype == LPMGPU_ELASTIC_DAMAGE)
    {
        volatile double zero = 0.0;
        const double ddot_nonlocal = ddot_nl ? ddot_nl[i] : zero / zero;
        double d = damage[i] + ddot_nonlocal;
        if (d >= threshold)
            d = 1;
        damage[i] = d;
        changed = fabs(d - damage_last[i]) > 1e-3;
    }
    else
    {
        for (int b = bstart[i]; b < bstart[i + 1]; ++b)
            if (bstrain[b] >= critical && fabs(bdamage[b] - 1.0) > kEps)
            {
                changed = true;
                bdamage[b] = 1;
            }
    }
    if (changed)
        atomicExch(&scal->any_flag, 1);
}

cudaError_t launch_static_damage(Problem &p)
{
    cudaError_t e = cudaMemsetAsync(&p.scal->any_flag, 0, sizeof(int), p.stream);
    if (e != cudaSuccess)
        return e;
    // fatigue particles keep Particle::updateParticleStaticDamage, which changes nothing
    // (particle.h:63): their damage moves only in SolverFatigue::updateFatigueDamage
    if (p.desc.ptype == LPMGPU_FATIGUE_HCF)
        return cudaSuccess;
    if (p.desc.ptype != LPMGPU_ELASTIC && (e = launch_nonlocal_average(p)) != cudaSuccess)
        return e;
    // damage_threshold is never assigned for J2 (particle_j2plasticity.h:22): 0
    const double threshold = (p.desc.ptype == LPMGPU_ELASTIC_DAMAGE) ? p.desc.damage_threshold : 0.0;
    k_static_damage<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.desc.ptype, p.desc.undamaged_type,
                                                            p.desc.critical_bstrain, threshold, p.type, p.bstart,
                                                            p.bstrain, p.ddot_nonlocal, p.bdamage, p.damage,
                                                            p.damage_last, p.scal);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// Solver::solveLinearSystem position update (solver.h:101-108)
__global__ void k_add_disp(int n, int dim, const double *__restrict__ x, double *__restrict__ xyz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    for (int k = 0; k < dim; ++k)
        xyz[3 * i + k] = xyz[3 * i + k] + (0.0 + x[(int64_t)dim * i + k]);
}

cudaError_t launch_add_disp(Problem &p)
{
    k_add_disp<<<div_up(p.n, 256), 256, 0, p.stream>>>(p.n, p.dim, p.x, p.xyz);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

__global__ void k_force_bc(int count, const int *__restrict__ ids, double fx, double fy, double fz,
                           double *__restrict__ pex)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count)
        return;
    const int i = ids[q];
    pex[3 * i] += fx / count;
    pex[3 * i + 1] += fy / count;
    pex[3 * i + 2] += fz / count;
}

__global__ void k_disp_bc(int count, const int *__restrict__ ids, int flag, double step, double *__restrict__ xyz,
                          int *__restrict__ cons)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count)
        return;
    const int i = ids[q];
    xyz[3 * i + flag] = xyz[3 * i + flag] + step;
    cons[3 * i + flag] = 1;
}

// updateForceBC then updateDisplacementBC, each BC in order.  A particle that appears twice in
// one group would be updated by two threads; the reference's groups hold distinct particles.
cudaError_t launch_apply_bc(Problem &p, const lpmgpu_load_step &s)
{
    size_t total = 0;
    for (int f = 0; f < s.nforce; ++f)
        total += (size_t)s.force[f].count;
    for (int d = 0; d < s.ndisp; ++d)
        total += (size_t)s.disp[d].count;
    if (total == 0)
        return cudaSuccess;
    int *dids = nullptr;
    cudaError_t e = cudaMallocAsync(&dids, sizeof(int) * total, p.stream);
    if (e != cudaSuccess)
        return e;
    std::vector<int> h(total);
    size_t o = 0;
    for (int f = 0; f < s.nforce; ++f)
        for (int q = 0; q < s.force[f].count; ++q)
            h[o++] = s.force[f].ids[q];
    for (int d = 0; d < s.ndisp; ++d)
        for (int q = 0; q < s.disp[d].count; ++q)
            h[o++] = s.disp[d].ids[q];
    e = cudaMemcpyAsync(dids, h.data(), sizeof(int) * total, cudaMemcpyHostToDevice, p.stream);
    o = 0;
    for (int f = 0; f < s.nforce && e == cudaSuccess; ++f)
    {
        const auto &b = s.force[f];
        if (b.count > 0)
        {
            k_force_bc<<<div_up(b.count, 256), 256, 0, p.stream>>>(b.count, dids + o, b.fx, b.fy, b.fz, p.pex);
            p.ctr.kernel_launches++;
        }
        o += b.count;
    }
    for (int d = 0; d < s.ndisp && e == cudaSuccess; ++d)
    {
        const auto &b = s.disp[d];
        if (b.count > 0)
        {
            k_disp_bc<<<div_up(b.count, 256), 256, 0, p.stream>>>(b.count, dids + o, b.flag, b.step, p.xyz, p.cons);
            p.ctr.kernel_launches++;
        }
        o += b.count;
    }
    if (e == cudaSuccess)
        e = cudaGetLastError();
    // the host vector must outlive the async copy
    cudaError_t s2 = cudaStreamSynchronize(p.stream);
    cudaFreeAsync(dids, p.stream);
    return e != cudaSuccess ? e : s2;
}

} // namespace lpm
