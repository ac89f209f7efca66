// Per-step text output in the reference's LAMMPS dump format: Assembly::writeDump
// (include/assembly.h:310-335), which SolverStatic::solveProblem calls after every load step
// (include/solver_static.h:89).
//
// The formatter is host code: the particles are split into contiguous chunks, each chunk is
// formatted by its own thread with the reference's printf conversions (so the bytes are those
// the reference writes for the same values), and the chunks are appended in order.  For a device
// problem the step's fields are copied into pinned host buffers on the handle's stream, after
// its pending work; with async = 1 a writer thread of the handle formats and appends the step
// while the caller goes on with the next load step.
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "lpm_internal.cuh"

namespace lpm
{

struct DumpFields
{
    int n = 0, nsv = 1;
    const int *type = nullptr;
    const double *xyz = nullptr, *xyz0 = nullptr, *stress = nullptr, *damage = nullptr, *dv = nullptr,
                 *sv = nullptr;
};

// particles [lo, hi) as the reference's per-particle lines (assembly.h:326-331)
static void format_rows(const DumpFields &f, int lo, int hi, std::string &out)
{
    char line[512];
    out.clear();
    out.reserve((size_t)(hi - lo) * 192);
    for (int i = lo; i < hi; ++i)
    {
        const double *x = f.xyz + 3 * (size_t)i, *x0 = f.xyz0 + 3 * (size_t)i, *s = f.stress + 6 * (size_t)i;
        const int len = std::snprintf(
            line, sizeof line,
            "%d %d %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e %.4e\n", i,
            f.type ? f.type[i] : 0, x[0], x[1], x[2], x[0] - x0[0], x[1] - x0[1], x[2] - x0[2], s[0], s[1], s[2],
            s[3], s[4], s[5], f.damage[i], f.dv[i], f.sv[(size_t)f.nsv * i]);
        out.append(line, (size_t)std::min(len, (int)sizeof line - 1));
    }
}

// Appends one step to path ("a+", as the reference opens it).  threads <= 0: all host cores.
static int32_t write_dump(const char *path, int step, const double box[6], const DumpFields &f, int threads)
{
    int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    T = std::max(1, std::min(T, (f.n + 4095) / 4096)); // at least 4096 particles per thread
    std::vector<std::string> parts(T);
    auto work = [&](int k) {
        const int lo = (int)((int64_t)f.n * k / T), hi = (int)((int64_t)f.n * (k + 1) / T);
        format_rows(f, lo, hi, parts[k]);
    };
    std::vector<std::thread> th;
    for (int k = 1; k < T; ++k)
        th.emplace_back(work, k);
    work(0);
    for (auto &t : th)
        t.join();
    FILE *fp = std::fopen(path, "a+");
    if (!fp)
    {
        set_last_error(std::string("dump: cannot open ") + path);
        return LPMGPU_ERR_INVALID_ARG;
    }
    // the header of assembly.h:314-324
    std::fprintf(fp, "ITEM: TIMESTEP\n");
    std::fprintf(fp, "%d\n", step);
    std::fprintf(fp, "ITEM: NUMBER OF ATOMS\n");
    std::fprintf(fp, "%d\n", f.n);
    std::fprintf(fp, "ITEM: BOX BOUNDS pp pp pp\n");
    std::fprintf(fp, "%8.8f %8.8f\n", box[0], box[1]);
    std::fprintf(fp, "%8.8f %8.8f\n", box[2], box[3]);
    std::fprintf(fp, "%8.8f %8.8f\n", box[4], box[5]);
    std::fprintf(fp, "ITEM: ATOMS id type x y z dx dy dz s11 s22 s33 s23 s13 s12 damage damage_visual state_var[0] \n");
    bool ok = true;
    for (const auto &s : parts)
        ok = ok && std::fwrite(s.data(), 1, s.size(), fp) == s.size();
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok)
    {
        set_last_error(std::string("dump: write failed on ") + path);
        return LPMGPU_ERR_INVALID_ARG;
    }
    return LPMGPU_OK;
}

// One queued step: its fields in pinned host memory and the event that marks their arrival.
struct DumpJob
{
    std::string path;
    int step = 0, threads = 0;
    double box[6] = {0, 0, 0, 0, 0, 0};
    double *buf = nullptr; // xyz 3n | stress 6n | damage n | damage_visual n | state_var nsv*n
    cudaEvent_t ev = nullptr;
};

// The writer of one handle: at most kSlots steps in flight, written in the order queued.
struct DumpWriter
{
    static constexpr int kSlots = 2;
    int device = 0, n = 0, nsv = 1;
    const double *xyz0 = nullptr;
    const int *type = nullptr;
    std::vector<DumpJob *> jobs, free_jobs;
    std::deque<DumpJob *> queue;
    int busy = 0; // jobs queued or being written
    bool stop = false;
    int32_t err = LPMGPU_OK;
    std::string errmsg;
    std::mutex mu;
    std::condition_variable cv;
    std::thread th;

    DumpFields fields(const DumpJob &j) const
    {
        DumpFields f;
        f.n = n;
        f.nsv = nsv;
        f.type = type;
        f.xyz0 = xyz0;
        f.xyz = j.buf;
        f.stress = j.buf + 3 * (size_t)n;
        f.damage = j.buf + 9 * (size_t)n;
        f.dv = j.buf + 10 * (size_t)n;
        f.sv = j.buf + 11 * (size_t)n;
        return f;
    }

    void run()
    {
        cudaSetDevice(device);
        for (;;)
        {
            DumpJob *j = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty())
                    return;
                j = queue.front();
                queue.pop_front();
            }
            int32_t r = LPMGPU_OK;
            const cudaError_t e = cudaEventSynchronize(j->ev);
            if (e != cudaSuccess)
            {
                set_last_error(std::string("dump: ") + cudaGetErrorString(e));
                r = LPMGPU_ERR_CUDA;
            }
            else
                r = write_dump(j->path.c_str(), j->step, j->box, fields(*j), j->threads);
            {
                std::lock_guard<std::mutex> lk(mu);
                if (r != LPMGPU_OK && err == LPMGPU_OK)
                {
                    err = r;
                    errmsg = lpmgpu_last_error();
                }
                free_jobs.push_back(j);
                busy--;
            }
            cv.notify_all();
        }
    }

    // a free job (allocated on first use, at most kSlots), waiting for one when all are taken
    int32_t take(DumpJob **out)
    {
        std::unique_lock<std::mutex> lk(mu);
        if (free_jobs.empty() && (int)jobs.size() < kSlots)
        {
            auto *j = new DumpJob();
            const size_t bytes = sizeof(double) * (size_t)n * (11 + nsv);
            cudaError_t e = cudaMallocHost(&j->buf, bytes);
            if (e == cudaSuccess)
                e = cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming);
            if (e != cudaSuccess)
            {
                if (j->buf)
                    cudaFreeHost(j->buf);
                delete j;
                set_last_error(std::string("dump: ") + cudaGetErrorString(e));
                return e == cudaErrorMemoryAllocation ? LPMGPU_ERR_OUT_OF_MEMORY : LPMGPU_ERR_CUDA;
            }
            jobs.push_back(j);
            free_jobs.push_back(j);
        }
        cv.wait(lk, [&] { return !free_jobs.empty(); });
        *out = free_jobs.back();
        free_jobs.pop_back();
        return LPMGPU_OK;
    }

    void submit(DumpJob *j)
    {
        {
            std::lock_guard<std::mutex> lk(mu);
            queue.push_back(j);
            busy++;
            if (!th.joinable())
                th = std::thread(&DumpWriter::run, this);
        }
        cv.notify_all();
    }

    void give_back(DumpJob *j)
    {
        std::lock_guard<std::mutex> lk(mu);
        free_jobs.push_back(j);
    }

    int32_t flush()
    {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return busy == 0; });
        const int32_t r = err;
        if (r != LPMGPU_OK)
            set_last_error(errmsg);
        err = LPMGPU_OK;
        errmsg.clear();
        return r;
    }

    ~DumpWriter()
    {
        flush();
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (th.joinable())
            th.join();
        cudaSetDevice(device);
        for (DumpJob *j : jobs)
        {
            cudaEventDestroy(j->ev);
            cudaFreeHost(j->buf);
            delete j;
        }
    }
};

void release_dump_writer(Problem &p)
{
    delete static_cast<DumpWriter *>(p.dump);
    p.dump = nullptr;
}

} // namespace lpm

using namespace lpm;

extern "C" int32_t lpmgpu_format_dump(const char *path, int32_t step, int32_t n, const int32_t *type,
                                      const double box[6], const double *xyz, const double *xyz_initial,
                                      const double *stress, const double *damage, const double *damage_visual,
                                      const double *state_var, int32_t nsv, int32_t threads)
{
    if (!path || n < 0 || !box || nsv < 1 || (n > 0 && (!xyz || !xyz_initial || !stress || !damage ||
                                                        !damage_visual || !state_var)))
        return LPMGPU_ERR_INVALID_ARG;
    DumpFields f;
    f.n = n;
    f.nsv = nsv;
    f.type = type;
    f.xyz = xyz;
    f.xyz0 = xyz_initial;
    f.stress = stress;
    f.damage = damage;
    f.dv = damage_visual;
    f.sv = state_var;
    return write_dump(path, step, box, f, threads);
}

extern "C" int32_t lpmgpu_dump_write(lpmgpu_solver *h, const char *path, int32_t step, const double box[6],
                                     int32_t threads, int32_t async)
{
    if (!h || !path || !box)
        return LPMGPU_ERR_INVALID_ARG;
    Problem &p = h->p;
    cudaError_t e = cudaSetDevice(p.device);
    if (e != cudaSuccess)
    {
        set_last_error(std::string("dump: ") + cudaGetErrorString(e));
        return LPMGPU_ERR_CUDA;
    }
    if (!p.dump)
    {
        auto *w = new DumpWriter();
        w->device = p.device;
        w->n = p.n;
        w->nsv = p.nsv;
        w->xyz0 = p.xyz0_host.data();
        w->type = p.type_host.data();
        p.dump = w;
    }
    auto *w = static_cast<DumpWriter *>(p.dump);
    DumpJob *j = nullptr;
    int32_t r = w->take(&j);
    if (r != LPMGPU_OK)
        return r;
    j->path = path;
    j->step = step;
    j->threads = threads;
    std::memcpy(j->box, box, sizeof j->box);
    const size_t n = p.n;
    const std::pair<const double *, size_t> src[] = {
        {p.xyz, 3 * n}, {p.stress, 6 * n}, {p.damage, n}, {p.damage_visual, n}, {p.sv, (size_t)p.nsv * n}};
    size_t off = 0;
    for (const auto &s : src)
    {
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(j->buf + off, s.first, sizeof(double) * s.second, cudaMemcpyDeviceToHost, p.stream);
        off += s.second;
    }
    if (e == cudaSuccess)
        e = cudaEventRecord(j->ev, p.stream);
    if (e != cudaSuccess)
    {
        w->give_back(j);
        set_last_error(std::string("dump: ") + cudaGetErrorString(e));
        return LPMGPU_ERR_CUDA;
    }
    w->submit(j);
    return async ? LPMGPU_OK : w->flush();
}

extern "C" int32_t lpmgpu_dump_flush(lpmgpu_solver *h)
{
    if (!h)
        return LPMGPU_ERR_INVALID_ARG;
    if (!h->p.dump)
        return LPMGPU_OK;
    return static_cast<DumpWriter *>(h->p.dump)->flush();
}
