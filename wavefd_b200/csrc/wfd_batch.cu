// Batched shots: many 3D propagator objects (ginsu windows of one survey model, uneven sizes, Iso,
// VTI and TTI mixed) advanced together. The reference has no batching (Ginsu is exported by
// src/WaveFD.jl:52 but not defined; its tile knobs nbx/nby/nbz and tilesize() are per object,
// src/prop3DAcoIsoDenQ_DEO2_FDTD.jl:10-12, :159-185); this is designed from scratch.
//
// One persistent launch per physics class advances every shot of that class by one time step:
// work items are (shot, x-chunk, tile) triples; a descriptor per shot and pointer parity holds its
// sizes, output arrays and tensor maps in device memory, and CTAs take items from a counter in the
// order the planner packed them. The step arithmetic is the single-object kernels' own, so every
// shot's wavefields are bitwise those of stepping the objects one by one.
// After the step(s), one launch injects every shot's source samples and one extracts every
// shot's receiver samples (the grouped, ordered accumulation of spacetime.cc:144-204); the time
// index lives in device memory and is advanced by the graph itself, so a pair of steps is
// captured once in a CUDA graph and replayed for the whole time loop.
// The planner's knobs (x-chunk length, i.e. the tile's extent along the sweep; item order; the
// class launches concurrent or serial) are picked by an autotuner that times candidate launches
// on the batch's own arrays and restores what they overwrote.
#include <float.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "wavefd_b200.h"
#include "wfd_alloc.h"
#include "wfd_points.h"
#include "wfd_prop.h"

namespace wfd {

namespace {

// ---- kernels ---------------------------------------------------------------------------------------
// extract = 0: field[key] (+)= sum c * data[other*nt + it-1] (injection); extract = 1:
// data[key*nt + it-1] (+)= sum c * field[other] (extraction). Separate IEEE multiply and add in
// group order, as the single-shot tables do. Shots whose trace length is below it are skipped.
__global__ void k_batch_points(long ngroups, const int *__restrict__ gshot, const long *__restrict__ key,
                               const long *__restrict__ start, const long *__restrict__ other,
                               const float *__restrict__ c, float *const *__restrict__ fieldp,
                               float *const *__restrict__ datap, const long *__restrict__ ntv,
                               const long *__restrict__ d_it, int extract) {
    const long gi = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= ngroups) return;
    const int s = gshot[gi];
    const long it = *d_it, nt = ntv[s];
    if (it < 1 || it > nt) return;
    float *field = fieldp[s];
    float *data = datap[s];
    float *dst = extract ? data + key[gi] * nt + (it - 1) : field + key[gi];
    float acc = *dst;
    for (long j = start[gi]; j < start[gi + 1]; j++) {
        const float v = extract ? field[other[j]] : data[other[j] * nt + (it - 1)];
        acc = __fadd_rn(acc, __fmul_rn(c[j], v));
    }
    *dst = acc;
}

__global__ void k_tick(long *it) { *it += 1; }

// shot[x,y,z] = survey[x0+x, y0+y, z0+z], indices clamped to the survey (edge extension)
__global__ void k_crop(const float *__restrict__ survey, long snx, long sny, long snz, long x0, long y0, long z0,
                       float *__restrict__ shot, long nx, long ny, long nz) {
    const long n = nx * ny * nz;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const long z = k % nz, r = k / nz, y = r % ny, x = r / ny;
        const long sx = min(max(x0 + x, 0L), snx - 1), sy = min(max(y0 + y, 0L), sny - 1),
                   sz = min(max(z0 + z, 0L), snz - 1);
        shot[k] = survey[(sx * sny + sy) * snz + sz];
    }
}

// survey[x0+x, y0+y, z0+z] += shot[x,y,z] where inside the survey
__global__ void k_accumulate(float *__restrict__ survey, long snx, long sny, long snz, long x0, long y0, long z0,
                             const float *__restrict__ shot, long nx, long ny, long nz) {
    const long n = nx * ny * nz;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const long z = k % nz, r = k / nz, y = r % ny, x = r / ny;
        const long sx = x0 + x, sy = y0 + y, sz = z0 + z;
        if (sx < 0 || sx >= snx || sy < 0 || sy >= sny || sz < 0 || sz >= snz) continue;
        float *d = survey + (sx * sny + sy) * snz + sz;
        *d = __fadd_rn(*d, shot[k]);
    }
}

// ---- host objects ----------------------------------------------------------------------------------
struct Plan {
    int xtarget = 128;  // x-chunk length target (0: whole nx)
    int order = 0;      // 0: longest items first, 1: shots interleaved
};

struct Group {
    int phys = ISO;
    std::vector<int> shots;  // batch shot indices
    Plan plan;
    std::vector<int> xchunk;
    void *d_desc = nullptr;  // 2 descriptors per shot (pointer parities 0 and 1)
    int *d_sel = nullptr;    // [2][nshots]: descriptor index per shot for the two steps of a pair
    int2 *d_items = nullptr;
    int nitems = 0, grid = 0, grid_cap = 0, warmup = 0;
    size_t desc_size() const { return phys == ISO ? sizeof(IsoShotDesc) : sizeof(AnisoShotDesc); }
};

struct Acq {
    std::vector<PointsT<float>> src, rec;
    const float *wavelet = nullptr;
    float *traces = nullptr;
    long nt = 0;
};

struct PointSet {
    long ngroups = 0;
    int *d_shot = nullptr;
    long *d_key = nullptr, *d_start = nullptr, *d_other = nullptr;
    float *d_c = nullptr;
};

struct Batch {
    std::vector<Prop *> props;
    std::vector<float *> baseP, baseO, baseM, baseMO;  // pCur/pOld/mCur/mOld at creation (parity 0)
    int device = 0;
    bool strict = false;
    Grid gc{};
    cudaStream_t stream = nullptr, side[3] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[3] = {}, ev_t0 = nullptr, ev_t1 = nullptr;
    Group groups[3];
    int *d_counter = nullptr;  // one per group
    long *d_it = nullptr;
    int mode = 0;  // 0: class launches concurrent, 1: serial
    std::vector<Acq> acq;
    bool acq_dirty = true;
    PointSet src, rec;
    float **d_fieldp = nullptr;  // [2][nshots]: pCur after step k of a pair
    float **d_datap = nullptr;   // [2][nshots]: wavelet, traces
    long *d_nt = nullptr;
    std::vector<int> par_uploaded;  // parities the device tables were built for
    cudaGraphExec_t exec = nullptr;
    bool graph_dirty = true;
    int status = WFD_OK;
    std::string message;
    bool tuned = false;
    std::vector<float> tune_ms;  // best ms per group and the chosen mode's step
};

int bfail(Batch *b, int code, const std::string &msg) {
    b->status = code;
    b->message = msg;
    set_global_error(code, msg);
    return code;
}

int bcheck(Batch *b, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return WFD_OK;
    return bfail(b, WFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void free_pointset(PointSet &p) {
    cudaFree(p.d_shot);
    cudaFree(p.d_key);
    cudaFree(p.d_start);
    cudaFree(p.d_other);
    cudaFree(p.d_c);
    p = PointSet{};
}

int parity(const Batch *b, int s) { return b->props[s]->field[F_PCUR] == b->baseP[s] ? 0 : 1; }

Fields fields_at(const Batch *b, int s, int par) {
    Fields F = b->props[s]->fields();
    F.pcur = par ? b->baseO[s] : b->baseP[s];
    F.pold = par ? b->baseP[s] : b->baseO[s];
    if (b->props[s]->phys != ISO) {
        F.mcur = par ? b->baseMO[s] : b->baseM[s];
        F.mold = par ? b->baseM[s] : b->baseMO[s];
    }
    return F;
}

bool describe(const Batch *b, int phys, const Grid &g, const Fields &F, int xchunk, void *d, TileInfo *t) {
    if (phys == ISO)
        return b->strict ? wfd_strict::iso3d_tma_describe(g, F, xchunk, (IsoShotDesc *)d, t)
                         : wfd_fast::iso3d_tma_describe(g, F, xchunk, (IsoShotDesc *)d, t);
    return b->strict ? wfd_strict::aniso3d_tma_describe(g, phys, F, xchunk, (AnisoShotDesc *)d, t)
                     : wfd_fast::aniso3d_tma_describe(g, phys, F, xchunk, (AnisoShotDesc *)d, t);
}

// Work items of a group under its plan: x-chunks per shot, then the item order.
int plan_group(Batch *b, Group &G) {
    const int ns = (int)G.shots.size();
    if (!ns) return WFD_OK;
    TileInfo t{};
    describe(b, G.phys, b->props[G.shots[0]]->grid(), b->props[G.shots[0]]->fields(), 1, nullptr, &t);
    G.grid_cap = t.grid_cap;
    G.warmup = t.warmup;
    G.xchunk.assign(ns, 1);
    struct Item {
        int shot, local;
        long cost;
    };
    std::vector<Item> items;
    std::vector<std::vector<Item>> per(ns);
    for (int i = 0; i < ns; i++) {
        const Prop *p = b->props[G.shots[i]];
        const long nx = p->nx;
        const int nch = G.plan.xtarget > 0 ? (int)std::max(1L, (nx + G.plan.xtarget - 1) / G.plan.xtarget) : 1;
        const int xc = (int)((nx + nch - 1) / nch);
        G.xchunk[i] = xc;
        const int nchr = (int)((nx + xc - 1) / xc);
        const int ntz = (int)((p->nz + t.tz - 1) / t.tz), nty = (int)((p->ny + t.ty - 1) / t.ty);
        for (int ch = 0; ch < nchr; ch++) {
            const long len = std::min<long>(xc, nx - (long)ch * xc);
            for (int l = 0; l < ntz * nty; l++) per[i].push_back({i, ch * ntz * nty + l, len + t.warmup});
        }
    }
    if (G.plan.order == 0) {
        for (auto &v : per) items.insert(items.end(), v.begin(), v.end());
        std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &c) { return a.cost > c.cost; });
    } else {
        size_t longest = 0;
        for (auto &v : per) longest = std::max(longest, v.size());
        for (size_t r = 0; r < longest; r++)
            for (int i = 0; i < ns; i++)
                if (r < per[i].size()) items.push_back(per[i][r]);
    }
    // descriptors for both pointer parities
    const size_t dsz = G.desc_size();
    std::vector<unsigned char> host(dsz * 2 * ns);
    for (int i = 0; i < ns; i++) {
        const int s = G.shots[i];
        const Grid g = b->props[s]->grid();
        for (int par = 0; par < 2; par++)
            if (!describe(b, G.phys, g, fields_at(b, s, par), G.xchunk[i], host.data() + dsz * (2 * i + par), nullptr))
                return bfail(b, WFD_ERR_UNSUPPORTED, "tensor maps of a shot could not be encoded");
    }
    std::vector<int2> hitems(items.size());
    for (size_t k = 0; k < items.size(); k++) hitems[k] = make_int2(items[k].shot, items[k].local);
    // launches already queued may still read the old tables
    if (int rc = bcheck(b, cudaStreamSynchronize(b->stream), "plan")) return rc;
    cudaFree(G.d_desc);
    cudaFree(G.d_items);
    G.d_desc = nullptr;
    G.d_items = nullptr;
    if (int rc = bcheck(b, wfd::dMalloc(&G.d_desc, host.size()), "descriptor allocation")) return rc;
    if (int rc = bcheck(b, wfd::dMalloc(&G.d_items, sizeof(int2) * hitems.size()), "item allocation")) return rc;
    if (!G.d_sel)
        if (int rc = bcheck(b, wfd::dMalloc(&G.d_sel, sizeof(int) * 2 * ns), "selector allocation")) return rc;
    cudaMemcpy(G.d_desc, host.data(), host.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(G.d_items, hitems.data(), sizeof(int2) * hitems.size(), cudaMemcpyHostToDevice);
    G.nitems = (int)hitems.size();
    G.grid = std::min(G.nitems, G.grid_cap);
    b->par_uploaded.clear();  // selectors are rebuilt on the next run
    b->graph_dirty = true;
    return bcheck(b, cudaGetLastError(), "plan upload");
}

// Point tables of every shot, concatenated (groups of one shot stay in the single-shot order).
int build_pointset(Batch *b, PointSet &ps, bool receivers) {
    free_pointset(ps);
    std::vector<int> shot;
    std::vector<long> key, start, other;
    std::vector<float> c;
    long base = 0;
    for (size_t s = 0; s < b->acq.size(); s++) {
        const auto &pts = receivers ? b->acq[s].rec : b->acq[s].src;
        if (pts.empty()) continue;
        Table<float> t;
        build(t, pts, receivers ? 1 : 0);
        for (long g = 0; g < t.ngroups; g++) {
            shot.push_back((int)s);
            key.push_back(t.key[g]);
            start.push_back(base + t.start[g]);
        }
        other.insert(other.end(), t.other.begin(), t.other.end());
        c.insert(c.end(), t.c.begin(), t.c.end());
        base += t.npoints;
    }
    start.push_back(base);
    ps.ngroups = (long)key.size();
    if (!ps.ngroups) return WFD_OK;
    bool ok = wfd::dMalloc(&ps.d_shot, sizeof(int) * shot.size()) == cudaSuccess &&
              wfd::dMalloc(&ps.d_key, sizeof(long) * key.size()) == cudaSuccess &&
              wfd::dMalloc(&ps.d_start, sizeof(long) * start.size()) == cudaSuccess &&
              wfd::dMalloc(&ps.d_other, sizeof(long) * other.size()) == cudaSuccess &&
              wfd::dMalloc(&ps.d_c, sizeof(float) * c.size()) == cudaSuccess;
    if (!ok) return bfail(b, WFD_ERR_ALLOC, "point table allocation failed");
    cudaMemcpy(ps.d_shot, shot.data(), sizeof(int) * shot.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(ps.d_key, key.data(), sizeof(long) * key.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(ps.d_start, start.data(), sizeof(long) * start.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(ps.d_other, other.data(), sizeof(long) * other.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(ps.d_c, c.data(), sizeof(float) * c.size(), cudaMemcpyHostToDevice);
    return bcheck(b, cudaGetLastError(), "point table upload");
}

// Selectors and per-shot pointer tables for the current pointer parities (uploaded on change).
int sync_tables(Batch *b) {
    const int n = (int)b->props.size();
    std::vector<int> par(n);
    for (int s = 0; s < n; s++) par[s] = parity(b, s);
    if (!b->acq_dirty && par == b->par_uploaded) return WFD_OK;
    // launches already queued may still read the tables being replaced
    if (int rc = bcheck(b, cudaStreamSynchronize(b->stream), "table upload")) return rc;
    if (b->acq_dirty) {
        if (int rc = build_pointset(b, b->src, false)) return rc;
        if (int rc = build_pointset(b, b->rec, true)) return rc;
        std::vector<float *> datap(2 * n, nullptr);
        std::vector<long> nt(n, 0);
        for (int s = 0; s < n; s++) {
            datap[s] = const_cast<float *>(b->acq[s].wavelet);
            datap[n + s] = b->acq[s].traces;
            nt[s] = b->acq[s].nt;
        }
        cudaMemcpy(b->d_datap, datap.data(), sizeof(float *) * 2 * n, cudaMemcpyHostToDevice);
        cudaMemcpy(b->d_nt, nt.data(), sizeof(long) * n, cudaMemcpyHostToDevice);
        b->acq_dirty = false;
        b->graph_dirty = true;
    }
    for (auto &G : b->groups) {
        const int ns = (int)G.shots.size();
        if (!ns) continue;
        std::vector<int> sel(2 * ns);
        for (int i = 0; i < ns; i++)
            for (int k = 0; k < 2; k++) sel[k * ns + i] = 2 * i + ((par[G.shots[i]] + k) & 1);
        cudaMemcpy(G.d_sel, sel.data(), sizeof(int) * 2 * ns, cudaMemcpyHostToDevice);
    }
    // pCur after step k of a pair: the pOld of the parity that step ran at
    std::vector<float *> fp(2 * n);
    for (int s = 0; s < n; s++)
        for (int k = 0; k < 2; k++) fp[k * n + s] = ((par[s] + k) & 1) == 0 ? b->baseO[s] : b->baseP[s];
    cudaMemcpy(b->d_fieldp, fp.data(), sizeof(float *) * 2 * n, cudaMemcpyHostToDevice);
    b->par_uploaded = par;
    return bcheck(b, cudaGetLastError(), "selector upload");
}

void launch_group(Batch *b, int gi, int k, cudaStream_t s) {
    Group &G = b->groups[gi];
    const int ns = (int)G.shots.size();
    if (!ns) return;
    const int *sel = G.d_sel + k * ns;
    if (G.phys == ISO) {
        if (b->strict) wfd_strict::iso3d_tma_batch(b->gc, (IsoShotDesc *)G.d_desc, sel, G.d_items, G.nitems,
                                                   b->d_counter + gi, G.grid, s);
        else wfd_fast::iso3d_tma_batch(b->gc, (IsoShotDesc *)G.d_desc, sel, G.d_items, G.nitems, b->d_counter + gi,
                                       G.grid, s);
    } else {
        if (b->strict) wfd_strict::aniso3d_tma_batch(b->gc, G.phys, (AnisoShotDesc *)G.d_desc, sel, G.d_items,
                                                     G.nitems, b->d_counter + gi, G.grid, s);
        else wfd_fast::aniso3d_tma_batch(b->gc, G.phys, (AnisoShotDesc *)G.d_desc, sel, G.d_items, G.nitems,
                                         b->d_counter + gi, G.grid, s);
    }
}

int active_groups(const Batch *b) {
    int n = 0;
    for (auto &G : b->groups) n += !G.shots.empty();
    return n;
}

// Step k (0 or 1) of a pair: the class launches, then injection and extraction at the device time
// index, then the index advances.
void enqueue_step(Batch *b, int k) {
    cudaStream_t s = b->stream;
    cudaMemsetAsync(b->d_counter, 0, sizeof(int) * 3, s);
    if (b->mode == 0 && active_groups(b) > 1) {
        cudaEventRecord(b->ev_fork, s);
        for (int gi = 0; gi < 3; gi++) {
            if (b->groups[gi].shots.empty()) continue;
            cudaStreamWaitEvent(b->side[gi], b->ev_fork, 0);
            launch_group(b, gi, k, b->side[gi]);
            cudaEventRecord(b->ev_join[gi], b->side[gi]);
        }
        for (int gi = 0; gi < 3; gi++)
            if (!b->groups[gi].shots.empty()) cudaStreamWaitEvent(s, b->ev_join[gi], 0);
    } else {
        for (int gi = 0; gi < 3; gi++) launch_group(b, gi, k, s);
    }
    const int n = (int)b->props.size();
    if (b->src.ngroups)
        k_batch_points<<<(unsigned)((b->src.ngroups + 255) / 256), 256, 0, s>>>(
            b->src.ngroups, b->src.d_shot, b->src.d_key, b->src.d_start, b->src.d_other, b->src.d_c,
            b->d_fieldp + k * n, b->d_datap, b->d_nt, b->d_it, 0);
    if (b->rec.ngroups)
        k_batch_points<<<(unsigned)((b->rec.ngroups + 255) / 256), 256, 0, s>>>(
            b->rec.ngroups, b->rec.d_shot, b->rec.d_key, b->rec.d_start, b->rec.d_other, b->rec.d_c,
            b->d_fieldp + k * n, b->d_datap + n, b->d_nt, b->d_it, 1);
    k_tick<<<1, 1, 0, s>>>(b->d_it);
}

void swap_all(Batch *b) {
    for (Prop *p : b->props) {
        std::swap(p->field[F_PCUR], p->field[F_POLD]);
        std::swap(p->field[F_MCUR], p->field[F_MOLD]);
        p->steps++;
    }
}

int build_graph(Batch *b) {
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    if (int rc = bcheck(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture"))
        return rc;
    enqueue_step(b, 0);
    enqueue_step(b, 1);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (int rc = bcheck(b, e, "end capture")) return rc;
    e = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int rc = bcheck(b, e, "graph instantiation")) return rc;
    b->graph_dirty = false;
    return WFD_OK;
}

// the batch's stream waits for work queued on the objects' own streams, and the other way round
void order_after_props(Batch *b) {
    for (Prop *p : b->props) {
        cudaEventRecord(b->ev_t0, p->stream);
        cudaStreamWaitEvent(b->stream, b->ev_t0, 0);
    }
}
void order_props_after(Batch *b) {
    cudaEventRecord(b->ev_t1, b->stream);
    for (Prop *p : b->props) cudaStreamWaitEvent(p->stream, b->ev_t1, 0);
}

int batch_sync(Batch *b) {
    if (int rc = bcheck(b, cudaStreamSynchronize(b->stream), "batch synchronize")) return rc;
    if (wfd_fast::fused_status_and_clear() | wfd_strict::fused_status_and_clear())
        return bfail(b, WFD_ERR_TIMEOUT, "a batched step kernel timed out waiting for its tile loads");
    return WFD_OK;
}

int batch_run(Batch *b, long nsteps, long it0, bool graph) {
    if (b->status) return b->status;
    order_after_props(b);
    for (Prop *p : b->props) prefetch_touched(p, b->stream);
    if (int rc = sync_tables(b)) return rc;
    if (int rc = bcheck(b, cudaMemcpyAsync(b->d_it, &it0, sizeof(long), cudaMemcpyHostToDevice, b->stream),
                        "time index"))
        return rc;
    // the host value must outlive the copy
    if (int rc = bcheck(b, cudaStreamSynchronize(b->stream), "time index")) return rc;
    long done = 0;
    if (graph && nsteps >= 2) {
        if (b->graph_dirty)
            if (int rc = build_graph(b)) return rc;
        for (; done + 2 <= nsteps; done += 2) {
            if (int rc = bcheck(b, cudaGraphLaunch(b->exec, b->stream), "graph launch")) return rc;
            for (Prop *p : b->props) p->steps += 2;
        }
    }
    for (; done < nsteps; done++) {
        // single steps: the selectors of step k of a pair match the parity after k flips
        enqueue_step(b, (int)(done & 1));
        swap_all(b);
    }
    if (int rc = bcheck(b, cudaGetLastError(), "batch step launch")) return rc;
    order_props_after(b);
    return WFD_OK;
}

// ---- autotuner -----------------------------------------------------------------------------------------
// Arrays a step writes: pOld (mOld) in place and pSpace (mSpace).
std::vector<float *> written_arrays(const Batch *b, int s) {
    const Prop *p = b->props[s];
    std::vector<float *> v = {p->field[F_POLD], p->field[F_PSPACE]};
    if (p->phys != ISO) {
        v.push_back(p->field[F_MOLD]);
        v.push_back(p->field[F_MSPACE]);
    }
    return v;
}

float time_launches(Batch *b, int gi, int reps) {
    cudaStream_t s = b->stream;
    auto one = [&]() {
        if (gi >= 0) {
            cudaMemsetAsync(b->d_counter, 0, sizeof(int) * 3, s);
            launch_group(b, gi, 0, s);
        } else {
            // every class, in the batch's current mode (no injection: the acquisition is not touched)
            cudaMemsetAsync(b->d_counter, 0, sizeof(int) * 3, s);
            if (b->mode == 0 && active_groups(b) > 1) {
                cudaEventRecord(b->ev_fork, s);
                for (int g = 0; g < 3; g++) {
                    if (b->groups[g].shots.empty()) continue;
                    cudaStreamWaitEvent(b->side[g], b->ev_fork, 0);
                    launch_group(b, g, 0, b->side[g]);
                    cudaEventRecord(b->ev_join[g], b->side[g]);
                }
                for (int g = 0; g < 3; g++)
                    if (!b->groups[g].shots.empty()) cudaStreamWaitEvent(s, b->ev_join[g], 0);
            } else {
                for (int g = 0; g < 3; g++) launch_group(b, g, 0, s);
            }
        }
    };
    one();  // warm-up
    cudaEventRecord(b->ev_t0, s);
    for (int r = 0; r < reps; r++) one();
    cudaEventRecord(b->ev_t1, s);
    if (cudaEventSynchronize(b->ev_t1) != cudaSuccess) return 1e30f;
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev_t0, b->ev_t1);
    return ms / reps;
}

int batch_tune(Batch *b, int reps) {
    if (b->status) return b->status;
    order_after_props(b);
    for (Prop *p : b->props) prefetch_touched(p, b->stream);
    if (int rc = sync_tables(b)) return rc;
    const int n = (int)b->props.size();
    // save what the trial launches overwrite
    size_t total = 0;
    for (int s = 0; s < n; s++) total += written_arrays(b, s).size() * (size_t)b->props[s]->ncells();
    float *save = nullptr;
    if (int rc = bcheck(b, wfd::dMalloc(&save, sizeof(float) * total), "tuner save area")) return rc;
    auto copy_all = [&](bool out) {
        size_t off = 0;
        for (int s = 0; s < n; s++) {
            const size_t bytes = sizeof(float) * (size_t)b->props[s]->ncells();
            for (float *a : written_arrays(b, s)) {
                if (out) cudaMemcpyAsync(save + off, a, bytes, cudaMemcpyDeviceToDevice, b->stream);
                else cudaMemcpyAsync(a, save + off, bytes, cudaMemcpyDeviceToDevice, b->stream);
                off += bytes / sizeof(float);
            }
        }
    };
    copy_all(true);
    b->tune_ms.assign(4, 0.0f);
    for (int gi = 0; gi < 3; gi++) {
        Group &G = b->groups[gi];
        if (G.shots.empty()) continue;
        long maxnx = 0;
        for (int s : G.shots) maxnx = std::max(maxnx, b->props[s]->nx);
        std::vector<int> targets = {0};
        for (int t : {320, 256, 192, 160, 128, 96, 64, 48})
            if (t < maxnx) targets.push_back(t);
        Plan best = G.plan;
        float best_ms = 1e30f;
        for (int t : targets)
            for (int order = 0; order < 2; order++) {
                G.plan.xtarget = t;
                G.plan.order = order;
                if (int rc = plan_group(b, G)) {
                    cudaFree(save);
                    return rc;
                }
                if (int rc = sync_tables(b)) {
                    cudaFree(save);
                    return rc;
                }
                const float ms = time_launches(b, gi, reps);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = G.plan;
                }
            }
        G.plan = best;
        if (int rc = plan_group(b, G)) {
            cudaFree(save);
            return rc;
        }
        b->tune_ms[gi] = best_ms;
    }
    if (int rc = sync_tables(b)) {
        cudaFree(save);
        return rc;
    }
    if (active_groups(b) > 1) {
        float ms_mode[2];
        for (int m = 0; m < 2; m++) {
            b->mode = m;
            ms_mode[m] = time_launches(b, -1, reps);
        }
        b->mode = ms_mode[1] < ms_mode[0] ? 1 : 0;
        b->tune_ms[3] = std::min(ms_mode[0], ms_mode[1]);
    } else {
        for (int gi = 0; gi < 3; gi++) b->tune_ms[3] += b->tune_ms[gi];
    }
    copy_all(false);
    cudaStreamSynchronize(b->stream);
    cudaFree(save);
    b->graph_dirty = true;
    b->tuned = true;
    order_props_after(b);
    return batch_sync(b);
}

void batch_destroy(Batch *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto &G : b->groups) {
        cudaFree(G.d_desc);
        cudaFree(G.d_sel);
        cudaFree(G.d_items);
    }
    free_pointset(b->src);
    free_pointset(b->rec);
    cudaFree(b->d_counter);
    cudaFree(b->d_it);
    cudaFree(b->d_fieldp);
    cudaFree(b->d_datap);
    cudaFree(b->d_nt);
    for (int i = 0; i < 3; i++) {
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_t0) cudaEventDestroy(b->ev_t0);
    if (b->ev_t1) cudaEventDestroy(b->ev_t1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

Batch *batch_create(Prop *const *props, long n) {
    if (n < 1 || !props) {
        set_global_error(WFD_ERR_ARG, "WFD_Batch_Create: empty shot list");
        return nullptr;
    }
    const Prop *p0 = props[0];
    for (long i = 0; i < n; i++) {
        const Prop *p = props[i];
        if (!p) {
            set_global_error(WFD_ERR_ARG, "WFD_Batch_Create: null object");
            return nullptr;
        }
        if (p->ndim != 3 || p->nz % 4 != 0 || !p->fused) {
            set_global_error(WFD_ERR_UNSUPPORTED,
                             "WFD_Batch_Create: shots must be 3D objects with nz a multiple of 4 and fused kernels");
            return nullptr;
        }
        if (p->dx != p0->dx || p->dy != p0->dy || p->dz != p0->dz || p->dt != p0->dt || p->fs != p0->fs ||
            p->strict != p0->strict || p->device != p0->device) {
            set_global_error(WFD_ERR_ARG,
                             "WFD_Batch_Create: shots must share dx, dy, dz, dt, the free surface, the strict/fast "
                             "mode and the device");
            return nullptr;
        }
        for (long j = 0; j < i; j++)
            if (props[j] == p) {
                set_global_error(WFD_ERR_ARG, "WFD_Batch_Create: an object is listed twice");
                return nullptr;
            }
    }
    Batch *b = new Batch();
    b->device = p0->device;
    b->strict = p0->strict;
    b->gc = p0->grid();
    b->groups[0].phys = ISO;
    b->groups[1].phys = VTI;
    b->groups[2].phys = TTI;
    for (long i = 0; i < n; i++) {
        Prop *p = props[i];
        b->props.push_back(p);
        b->baseP.push_back(p->field[F_PCUR]);
        b->baseO.push_back(p->field[F_POLD]);
        b->baseM.push_back(p->field[F_MCUR]);
        b->baseMO.push_back(p->field[F_MOLD]);
        b->groups[p->phys].shots.push_back((int)i);
    }
    b->acq.resize(n);
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; i < 3 && ok; i++)
        ok = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreate(&b->ev_t0) == cudaSuccess && cudaEventCreate(&b->ev_t1) == cudaSuccess &&
         wfd::dMalloc(&b->d_counter, sizeof(int) * 3) == cudaSuccess &&
         wfd::dMalloc(&b->d_it, sizeof(long)) == cudaSuccess &&
         wfd::dMalloc(&b->d_fieldp, sizeof(float *) * 2 * n) == cudaSuccess &&
         wfd::dMalloc(&b->d_datap, sizeof(float *) * 2 * n) == cudaSuccess &&
         wfd::dMalloc(&b->d_nt, sizeof(long) * n) == cudaSuccess;
    if (!ok) {
        set_global_error(WFD_ERR_ALLOC, "WFD_Batch_Create: device resources");
        batch_destroy(b);
        return nullptr;
    }
    for (auto &G : b->groups)
        if (plan_group(b, G)) {
            set_global_error(b->status, b->message);
            batch_destroy(b);
            return nullptr;
        }
    return b;
}

}  // namespace
}  // namespace wfd

using wfd::Batch;

namespace {
Batch *B(void *p) { return reinterpret_cast<Batch *>(p); }
unsigned blocks_for(long n) { return (unsigned)std::min<long>((n + 255) / 256, 148L * 16); }
}  // namespace

extern "C" void *WFD_Batch_Create(void *const *props, long nprops) {
    return wfd::batch_create(reinterpret_cast<wfd::Prop *const *>(props), nprops);
}

extern "C" void WFD_Batch_Free(void *batch) { wfd::batch_destroy(B(batch)); }

extern "C" int WFD_Batch_Status(void *batch) { return batch ? B(batch)->status : WFD_ERR_ARG; }

extern "C" const char *WFD_Batch_Message(void *batch) { return batch ? B(batch)->message.c_str() : "null batch"; }

extern "C" int WFD_Batch_SetAcquisition(void *batch, long shot, const SourcePoint32 *src, long nsrc,
                                        const float *wavelet, const SourcePoint32 *rec, long nrec, float *traces,
                                        long nt) {
    Batch *b = B(batch);
    if (!b || shot < 0 || shot >= (long)b->props.size() || nsrc < 0 || nrec < 0 || nt < 0 ||
        (nsrc > 0 && (!src || !wavelet)) || (nrec > 0 && (!rec || !traces)))
        return WFD_ERR_ARG;
    if ((wavelet && !wfd::device_accessible(wavelet)) || (traces && !wfd::device_accessible(traces)))
        return wfd::bfail(b, WFD_ERR_ARG, "wavelet and traces must be device or managed memory");
    const long ncell = b->props[shot]->ncells();
    wfd::Acq &a = b->acq[shot];
    a.src.clear();
    a.rec.clear();
    for (long i = 0; i < nsrc; i++) {
        if (src[i].iu < 1 || src[i].iu > ncell || src[i].ir < 1) return WFD_ERR_ARG;
        a.src.push_back({src[i].iu, src[i].ir, src[i].c});
    }
    for (long i = 0; i < nrec; i++) {
        if (rec[i].iu < 1 || rec[i].iu > ncell || rec[i].ir < 1) return WFD_ERR_ARG;
        a.rec.push_back({rec[i].iu, rec[i].ir, rec[i].c});
    }
    a.wavelet = wavelet;
    a.traces = traces;
    a.nt = nt;
    b->acq_dirty = true;
    return WFD_OK;
}

extern "C" int WFD_Batch_Plan(void *batch, long xchunk_target, int order, int concurrent) {
    Batch *b = B(batch);
    if (!b || xchunk_target < 0 || order < 0 || order > 1) return WFD_ERR_ARG;
    for (auto &G : b->groups) {
        G.plan.xtarget = (int)xchunk_target;
        G.plan.order = order;
        if (int rc = wfd::plan_group(b, G)) return rc;
    }
    b->mode = concurrent ? 0 : 1;
    b->graph_dirty = true;
    return WFD_OK;
}

extern "C" int WFD_Batch_Tune(void *batch, int reps) {
    if (!batch || reps < 1) return WFD_ERR_ARG;
    return wfd::batch_tune(B(batch), reps);
}

extern "C" int WFD_Batch_Run(void *batch, long nsteps, long it0, int use_graph) {
    if (!batch || nsteps < 0) return WFD_ERR_ARG;
    return wfd::batch_run(B(batch), nsteps, it0, use_graph != 0);
}

extern "C" int WFD_Batch_Synchronize(void *batch) { return batch ? wfd::batch_sync(B(batch)) : WFD_ERR_ARG; }

extern "C" void *WFD_Batch_Stream(void *batch) { return batch ? (void *)B(batch)->stream : nullptr; }

extern "C" int WFD_Batch_Info(void *batch, long *info, long ninfo) {
    Batch *b = B(batch);
    if (!b || !info || ninfo < 16) return WFD_ERR_ARG;
    for (int gi = 0; gi < 3; gi++) {
        const auto &G = b->groups[gi];
        info[4 * gi + 0] = (long)G.shots.size();
        info[4 * gi + 1] = G.nitems;
        info[4 * gi + 2] = G.grid;
        info[4 * gi + 3] = G.shots.empty() ? 0 : G.plan.xtarget;
    }
    info[12] = b->mode;
    info[13] = b->groups[0].plan.order | (b->groups[1].plan.order << 1) | (b->groups[2].plan.order << 2);
    info[14] = wfd::active_groups(b) + (b->src.ngroups ? 1 : 0) + (b->rec.ngroups ? 1 : 0) + 1;  // kernels per step
    info[15] = b->tuned ? 1 : 0;
    return WFD_OK;
}

extern "C" int WFD_Ginsu_Crop(const float *survey, long snx, long sny, long snz, long x0, long y0, long z0,
                              float *shot, long nx, long ny, long nz, void *stream) {
    if (!survey || !shot || snx < 1 || sny < 1 || snz < 1 || nx < 1 || ny < 1 || nz < 1) return WFD_ERR_ARG;
    if (!wfd::device_accessible(survey) || !wfd::device_accessible(shot)) return WFD_ERR_ARG;
    wfd::k_crop<<<blocks_for(nx * ny * nz), 256, 0, (cudaStream_t)stream>>>(survey, snx, sny, snz, x0, y0, z0, shot,
                                                                            nx, ny, nz);
    return cudaGetLastError() == cudaSuccess ? WFD_OK : WFD_ERR_CUDA;
}

extern "C" int WFD_Ginsu_Accumulate(float *survey, long snx, long sny, long snz, long x0, long y0, long z0,
                                    const float *shot, long nx, long ny, long nz, void *stream) {
    if (!survey || !shot || snx < 1 || sny < 1 || snz < 1 || nx < 1 || ny < 1 || nz < 1) return WFD_ERR_ARG;
    if (!wfd::device_accessible(survey) || !wfd::device_accessible(shot)) return WFD_ERR_ARG;
    wfd::k_accumulate<<<blocks_for(nx * ny * nz), 256, 0, (cudaStream_t)stream>>>(survey, snx, sny, snz, x0, y0, z0,
                                                                                  shot, nx, ny, nz);
    return cudaGetLastError() == cudaSuccess ? WFD_OK : WFD_ERR_CUDA;
}
