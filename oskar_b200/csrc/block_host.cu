// Host-buffer form of the fused tensor-core block: the call a simulator's
// per-block driver makes (the role of oskar_interferometer_run_block,
// oskar/interferometer/src/oskar_interferometer_run_block.c:28-153, for
// point sources without smearing): copy the block's inputs from host memory,
// correlate every (time, channel) of the block on the GPU, copy the
// visibility block back (group by group, overlapping the later groups'
// computation). Device buffers are kept by the library per device and grown
// on demand; with page-locked host buffers the copies run at full link
// speed.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <utility>
#include <vector>

#include "common.cuh"
#include "xcorr_tc.cuh"

namespace oskb {
namespace {

struct DevBuf
{
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct BlockBuffers
{
    DevBuf E, sky, uvw, wl, vis;
    cudaStream_t copy = nullptr;       // visibility downloads
    std::vector<cudaEvent_t> events;   // one per group of the current call
};

BlockBuffers g_bufs[64];

int ensure(DevBuf& b, size_t bytes)
{
    if (b.bytes >= bytes) return 0;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    if (cudaMalloc(&b.ptr, bytes) != cudaSuccess)
    {
        set_last_error("block buffers", cudaGetLastError());
        return OSKB_ERR_MEMORY_ALLOC_FAILURE;
    }
    b.bytes = bytes;
    return 0;
}

int copy_in(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
    {
        set_last_error("block H2D", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}

}  // namespace
}  // namespace oskb

using namespace oskb;

extern "C" int oskb_run_block_tc_host(int casa, int num_sources,
        int num_stations, int num_times, int num_channels, const float* E,
        const double* l, const double* m, const double* n, const double* I,
        const double* Q, const double* U, const double* V,
        const double* station_uvw, const double* freqs_hz,
        double uv_min_lambda, double uv_max_lambda, double* vis,
        void* stream)
{
    if (num_sources < 0 || num_stations < 0 || num_times < 0 ||
            num_channels < 0)
        return OSKB_ERR_INVALID_ARGUMENT;
    if (num_times == 0 || num_channels == 0 || num_stations < 2) return 0;
    if (!vis || !station_uvw || !freqs_hz) return OSKB_ERR_INVALID_ARGUMENT;
    const size_t nbl = (size_t) num_stations * (num_stations - 1) / 2;
    const size_t vis_bytes = (size_t) num_times * num_channels * nbl * 64;
    cudaStream_t s = as_stream(stream);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return OSKB_ERR_INVALID_ARGUMENT;
    BlockBuffers& b = g_bufs[dev];
    int err = ensure(b.vis, vis_bytes);
    if (err) return err;
    if (num_sources == 0)
    {
        memset(vis, 0, vis_bytes);
        return 0;
    }
    if (!E || !l || !m || !n || !I || !Q || !U || !V)
        return OSKB_ERR_INVALID_ARGUMENT;
    const size_t e_bytes = (size_t) num_stations * num_sources * 8 *
            sizeof(float);
    const size_t sky_bytes = 7 * (size_t) num_sources * sizeof(double);
    const size_t uvw_bytes = (size_t) num_times * 3 * num_stations *
            sizeof(double);
    if ((err = ensure(b.E, e_bytes)) || (err = ensure(b.sky, sky_bytes)) ||
            (err = ensure(b.uvw, uvw_bytes)) ||
            (err = ensure(b.wl, num_channels * sizeof(double))))
        return err;
    double* sky = static_cast<double*>(b.sky.ptr);
    const double* src[7] = {l, m, n, I, Q, U, V};
    std::vector<double> wl(num_channels);
    for (int c = 0; c < num_channels; ++c) wl[c] = freqs_hz[c] / 299792458.0;
    if ((err = copy_in(b.E.ptr, E, e_bytes, s))) return err;
    for (int k = 0; k < 7; ++k)
        if ((err = copy_in(sky + (size_t) k * num_sources, src[k],
                num_sources * sizeof(double), s)))
            return err;
    if ((err = copy_in(b.uvw.ptr, station_uvw, uvw_bytes, s))) return err;
    if ((err = copy_in(b.wl.ptr, wl.data(), num_channels * sizeof(double),
            s)))
        return err;
    // The block is cleared, then accumulated, as the reference does. Each
    // group of (dump, channel) problems is downloaded on a copy stream as
    // soon as its contraction has finished, while later groups compute.
    cudaMemsetAsync(b.vis.ptr, 0, vis_bytes, s);
    if (!b.copy)
    {
        if (cudaStreamCreateWithFlags(&b.copy, cudaStreamNonBlocking) !=
                cudaSuccess)
            b.copy = nullptr;
    }
    struct Ctx
    {
        cudaStream_t s, copy;
        std::vector<cudaEvent_t>* events;
        double* host;
        const double* dev;
        size_t problem_bytes;
        bool failed;
    } ctx{s, b.copy, &b.events, vis, static_cast<const double*>(b.vis.ptr),
          nbl * 64, false};
    auto after = [](void* p, int p0, int np) {
        Ctx& c = *static_cast<Ctx*>(p);
        if (!c.copy) return;
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) !=
                cudaSuccess)
        {
            c.failed = true;
            return;
        }
        c.events->push_back(ev);
        cudaEventRecord(ev, c.s);
        cudaStreamWaitEvent(c.copy, ev, 0);
        const size_t off = (size_t) p0 * c.problem_bytes;
        if (cudaMemcpyAsync(reinterpret_cast<char*>(c.host) + off,
                reinterpret_cast<const char*>(c.dev) + off,
                (size_t) np * c.problem_bytes, cudaMemcpyDeviceToHost,
                c.copy) != cudaSuccess)
            c.failed = true;
    };
    err = tc::correlate_block(casa, num_sources, num_stations, num_times,
            num_channels, static_cast<const float*>(b.E.ptr), sky,
            sky + num_sources, sky + 2 * (size_t) num_sources,
            sky + 3 * (size_t) num_sources, sky + 4 * (size_t) num_sources,
            sky + 5 * (size_t) num_sources, sky + 6 * (size_t) num_sources,
            static_cast<const double*>(b.uvw.ptr),
            static_cast<const double*>(b.wl.ptr), uv_min_lambda,
            uv_max_lambda, static_cast<double*>(b.vis.ptr), nullptr, 0,
            stream, b.copy ? +after : nullptr, &ctx);
    bool failed = ctx.failed || err != 0;
    if (!err && !b.copy &&
            cudaMemcpyAsync(vis, b.vis.ptr, vis_bytes,
            cudaMemcpyDeviceToHost, s) != cudaSuccess)
        failed = true;
    // Both streams must drain before the host buffer is complete.
    const cudaError_t e1 = cudaStreamSynchronize(s);
    const cudaError_t e2 = b.copy ? cudaStreamSynchronize(b.copy) :
            cudaSuccess;
    for (cudaEvent_t ev : b.events) cudaEventDestroy(ev);
    b.events.clear();
    if (err) return err;
    if (failed || e1 != cudaSuccess || e2 != cudaSuccess)
    {
        set_last_error("block D2H", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Pipelined form: a plan with two slots of device buffers, so that the
// upload of block b + 1 (on a copy-in stream) overlaps the correlation of
// block b (compute stream), and block b's visibilities download group by
// group on a copy-out stream. The sky is uploaded once per plan; the
// contraction's workspace is the plan's own (one, as the compute stream
// runs one block at a time).
// The first block picks the contraction form by timing the candidates on
// its own data (integer square tiles, integer CTA pairs, FP16 wide tiles);
// each slot's compute work (clear, maxabs, per group prep + contraction) is
// then captured once into a CUDA graph and replayed for every later block
// of that slot; the downloads stay outside the graph (their host
// destinations change) and wait on event nodes the graph records after
// each group.
// ---------------------------------------------------------------------------
struct oskb_TcPlan
{
    int casa, num_src, num_st, num_times, num_channels;
    double uv_min, uv_max;
    size_t e_bytes, uvw_bytes, vis_bytes, problem_bytes;
    double *sky, *wl;
    void* ws;
    size_t ws_bytes;
    int form;                    // contraction form in use (tc::Form)
    bool tuned, use_graph;
    double tune_ms[3];           // integer square, integer pairs, FP16 wide
    int graph_launches;
    struct Slot
    {
        void *E, *uvw, *vis;
        cudaEvent_t uploaded, computed, downloaded;
        bool used;
        cudaGraphExec_t exec;
        std::vector<std::pair<int, int>> groups;   // (p0, np) of the graph
        std::vector<cudaEvent_t> group_events;     // recorded by the graph
    } slot[2];
    cudaStream_t in, compute, out;
    std::vector<cudaEvent_t> group_events;   // the eager (non-graph) path
    size_t next_event;
    int next_slot;
    bool failed;
};

namespace {

struct PlanHook
{
    oskb_TcPlan* p;
    int slot;
    double* host;
};

// Eager path: record an event after the group and download it at once.
void plan_after_group(void* ctx, int p0, int np)
{
    PlanHook& h = *static_cast<PlanHook*>(ctx);
    oskb_TcPlan* p = h.p;
    if (p->next_event == p->group_events.size())
    {
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) !=
                cudaSuccess)
        {
            p->failed = true;
            return;
        }
        p->group_events.push_back(ev);
    }
    cudaEvent_t ev = p->group_events[p->next_event++];
    cudaEventRecord(ev, p->compute);
    cudaStreamWaitEvent(p->out, ev, 0);
    const size_t off = (size_t) p0 * p->problem_bytes;
    if (cudaMemcpyAsync(reinterpret_cast<char*>(h.host) + off,
            static_cast<const char*>(p->slot[h.slot].vis) + off,
            (size_t) np * p->problem_bytes, cudaMemcpyDeviceToHost, p->out)
            != cudaSuccess)
        p->failed = true;
}

// Capture path: the graph records one event per group; the downloads are
// enqueued after each replay.
void plan_capture_group(void* ctx, int p0, int np)
{
    PlanHook& h = *static_cast<PlanHook*>(ctx);
    oskb_TcPlan* p = h.p;
    oskb_TcPlan::Slot& s = p->slot[h.slot];
    const size_t g = s.groups.size();
    // an external event-record node: waited on outside the graph
    if (g >= s.group_events.size() ||
            cudaEventRecordWithFlags(s.group_events[g], p->compute,
            cudaEventRecordExternal) != cudaSuccess)
    {
        p->failed = true;
        return;
    }
    s.groups.emplace_back(p0, np);
}

int plan_correlate(oskb_TcPlan* p, int k, int form,
        void (*after)(void*, int, int), void* ctx)
{
    oskb_TcPlan::Slot& s = p->slot[k];
    const double* sky = p->sky;
    const size_t ns = p->num_src;
    if (cudaMemsetAsync(s.vis, 0, p->vis_bytes, p->compute) != cudaSuccess)
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    return tc::correlate_block(p->casa, p->num_src, p->num_st,
            p->num_times, p->num_channels, static_cast<const float*>(s.E),
            sky, sky + ns, sky + 2 * ns, sky + 3 * ns, sky + 4 * ns,
            sky + 5 * ns, sky + 6 * ns, static_cast<const double*>(s.uvw),
            p->wl, p->uv_min, p->uv_max, static_cast<double*>(s.vis), p->ws,
            p->ws_bytes, p->compute, after, ctx, nullptr, form);
}

// Times each candidate form on slot k's (uploaded) block and keeps the
// fastest; a candidate that fails is skipped.
int plan_tune(oskb_TcPlan* p, int k)
{
    static const int cand[3] = {tc::kFormI8, tc::kFormF16,
                                tc::kFormF16Wide};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess)
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    double best = 0.0;
    int best_form = tc::kFormDefault;
    for (int i = 0; i < 3; ++i)
    {
        p->tune_ms[i] = -1.0;
        cudaEventRecord(e0, p->compute);
        const int err = plan_correlate(p, k, cand[i], nullptr, nullptr);
        cudaEventRecord(e1, p->compute);
        if (cudaEventSynchronize(e1) != cudaSuccess || err)
        {
            cudaGetLastError();
            continue;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        p->tune_ms[i] = ms;
        if (best_form == tc::kFormDefault || ms < best)
        {
            best = ms;
            best_form = cand[i];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    p->form = best_form;
    p->tuned = true;
    return 0;
}

// Captures slot k's compute work into a graph; on failure the slot keeps
// running eagerly.
void plan_capture(oskb_TcPlan* p, int k)
{
    oskb_TcPlan::Slot& s = p->slot[k];
    s.groups.clear();
    if (tc::setup_device()) return;
    // one event per group at most one per problem, created before the
    // capture (no allocation inside it)
    const size_t num_problems = (size_t) p->num_times * p->num_channels;
    while (s.group_events.size() < num_problems)
    {
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) !=
                cudaSuccess)
            return;
        s.group_events.push_back(ev);
    }
    cudaError_t ce = cudaStreamBeginCapture(p->compute,
            cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess)
    {
        set_last_error("tc plan: begin capture", ce);
        cudaGetLastError();
        return;
    }
    PlanHook hook{p, k, nullptr};
    const bool failed_before = p->failed;
    const int err = plan_correlate(p, k, p->form, plan_capture_group,
            &hook);
    cudaGraph_t graph = nullptr;
    ce = cudaStreamEndCapture(p->compute, &graph);
    if (err || ce != cudaSuccess || !graph || p->failed != failed_before ||
            (ce = cudaGraphInstantiate(&s.exec, graph, 0)) != cudaSuccess)
    {
        char msg[160];
        snprintf(msg, sizeof(msg), "tc plan: capture of slot %d failed "
                "(correlate %d, capture status %d, hook %d); the slot runs "
                "without a graph", k, err, (int) ce,
                (int) (p->failed != failed_before));
        set_last_error_msg(msg);
        s.exec = nullptr;
        s.groups.clear();
        p->failed = failed_before;
        cudaGetLastError();
    }
    if (graph) cudaGraphDestroy(graph);
}

bool env_flag(const char* name, bool dflt)
{
    const char* e = getenv(name);
    return e ? atoi(e) != 0 : dflt;
}

}  // namespace

extern "C" {

void oskb_tc_plan_free(oskb_TcPlan* p)
{
    if (!p) return;
    if (p->in) cudaStreamSynchronize(p->in);
    if (p->compute) cudaStreamSynchronize(p->compute);
    if (p->out) cudaStreamSynchronize(p->out);
    for (auto& s : p->slot)
    {
        cudaFree(s.E); cudaFree(s.uvw); cudaFree(s.vis);
        if (s.uploaded) cudaEventDestroy(s.uploaded);
        if (s.computed) cudaEventDestroy(s.computed);
        if (s.downloaded) cudaEventDestroy(s.downloaded);
        if (s.exec) cudaGraphExecDestroy(s.exec);
        for (cudaEvent_t e : s.group_events) cudaEventDestroy(e);
    }
    for (cudaEvent_t e : p->group_events) cudaEventDestroy(e);
    cudaFree(p->sky); cudaFree(p->wl); cudaFree(p->ws);
    if (p->in) cudaStreamDestroy(p->in);
    if (p->compute) cudaStreamDestroy(p->compute);
    if (p->out) cudaStreamDestroy(p->out);
    delete p;
}

oskb_TcPlan* oskb_tc_plan_create(int casa, int num_sources, int num_stations,
        int num_times, int num_channels, const double* freqs_hz,
        double uv_min_lambda, double uv_max_lambda, int* status)
{
    if (*status) return nullptr;
    if (num_sources < 1 || num_stations < 2 || num_times < 1 ||
            num_channels < 1 || !freqs_hz)
    {
        *status = OSKB_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    oskb_TcPlan* p = new oskb_TcPlan();
    p->casa = casa; p->num_src = num_sources; p->num_st = num_stations;
    p->num_times = num_times; p->num_channels = num_channels;
    p->uv_min = uv_min_lambda; p->uv_max = uv_max_lambda;
    const size_t nbl = (size_t) num_stations * (num_stations - 1) / 2;
    p->problem_bytes = nbl * 64;
    p->vis_bytes = (size_t) num_times * num_channels * p->problem_bytes;
    p->e_bytes = (size_t) num_stations * num_sources * 8 * sizeof(float);
    p->uvw_bytes = (size_t) num_times * 3 * num_stations * sizeof(double);
    // an explicit form (OSKB_TC_PLAN_FORM = 1..5) skips the tuning
    const char* fe = getenv("OSKB_TC_PLAN_FORM");
    p->form = fe ? atoi(fe) : tc::kFormDefault;
    if (p->form < tc::kFormDefault || p->form > tc::kFormF16Pair ||
            p->form == 2)
        p->form = tc::kFormDefault;
    p->tuned = fe != nullptr || !env_flag("OSKB_TC_PLAN_TUNE", true);
    p->use_graph = env_flag("OSKB_TC_PLAN_GRAPH", true);
    for (double& t : p->tune_ms) t = -1.0;
    // workspace: up to 16 problems' operand images (the FP16 image, the
    // larger form), and no more than half the device memory free now
    const int num_problems = num_times * num_channels;
    const size_t one = oskb_correlate_block_tc_workspace_bytes(num_sources,
            num_stations, 1);
    const size_t img = one - oskb_correlate_block_tc_workspace_bytes(
            num_sources, num_stations, 0);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    size_t group = num_problems < 16 ? num_problems : 16;
    if (img && group > free_b / 2 / img) group = free_b / 2 / img;
    if (group < 1) group = 1;
    p->ws_bytes = oskb_correlate_block_tc_workspace_bytes(num_sources,
            num_stations, (int) group);
    bool ok = cudaStreamCreateWithFlags(&p->in, cudaStreamNonBlocking) ==
            cudaSuccess &&
            cudaStreamCreateWithFlags(&p->compute, cudaStreamNonBlocking) ==
            cudaSuccess &&
            cudaStreamCreateWithFlags(&p->out, cudaStreamNonBlocking) ==
            cudaSuccess &&
            cudaMalloc((void**) &p->sky, 7 * sizeof(double) * num_sources) ==
            cudaSuccess &&
            cudaMalloc((void**) &p->wl, sizeof(double) * num_channels) ==
            cudaSuccess &&
            cudaMalloc(&p->ws, p->ws_bytes) == cudaSuccess;
    for (auto& s : p->slot)
        ok = ok && cudaMalloc(&s.E, p->e_bytes) == cudaSuccess &&
                cudaMalloc(&s.uvw, p->uvw_bytes) == cudaSuccess &&
                cudaMalloc(&s.vis, p->vis_bytes) == cudaSuccess &&
                cudaEventCreateWithFlags(&s.uploaded,
                cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&s.computed,
                cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&s.downloaded,
                cudaEventDisableTiming) == cudaSuccess;
    if (ok)
    {
        std::vector<double> wl(num_channels);
        for (int c = 0; c < num_channels; ++c)
            wl[c] = freqs_hz[c] / 299792458.0;
        ok = cudaMemcpy(p->wl, wl.data(), sizeof(double) * num_channels,
                cudaMemcpyHostToDevice) == cudaSuccess;
    }
    if (!ok)
    {
        set_last_error("oskb_tc_plan_create", cudaGetLastError());
        oskb_tc_plan_free(p);
        *status = OSKB_ERR_MEMORY_ALLOC_FAILURE;
        return nullptr;
    }
    return p;
}

int oskb_tc_plan_set_sky(oskb_TcPlan* p, const double* l, const double* m,
        const double* n, const double* I, const double* Q, const double* U,
        const double* V)
{
    const double* src[7] = {l, m, n, I, Q, U, V};
    for (int k = 0; k < 7; ++k)
    {
        if (!src[k]) return OSKB_ERR_INVALID_ARGUMENT;
        if (cudaMemcpy(p->sky + (size_t) k * p->num_src, src[k],
                sizeof(double) * p->num_src, cudaMemcpyHostToDevice) !=
                cudaSuccess)
        {
            set_last_error("oskb_tc_plan_set_sky", cudaGetLastError());
            return OSKB_ERR_MEMORY_COPY_FAILURE;
        }
    }
    return 0;
}

int oskb_tc_plan_enqueue(oskb_TcPlan* p, const float* E_host,
        const double* station_uvw_host, double* vis_host)
{
    if (!E_host || !station_uvw_host || !vis_host)
        return OSKB_ERR_INVALID_ARGUMENT;
    const int k = p->next_slot;
    p->next_slot ^= 1;
    oskb_TcPlan::Slot& s = p->slot[k];
    // upload: the slot's E and uvw are free once its last block computed
    if (s.used) cudaStreamWaitEvent(p->in, s.computed, 0);
    if (cudaMemcpyAsync(s.E, E_host, p->e_bytes, cudaMemcpyHostToDevice,
            p->in) != cudaSuccess ||
            cudaMemcpyAsync(s.uvw, station_uvw_host, p->uvw_bytes,
            cudaMemcpyHostToDevice, p->in) != cudaSuccess)
    {
        set_last_error("oskb_tc_plan_enqueue", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    cudaEventRecord(s.uploaded, p->in);
    // compute: after the upload, and once the slot's visibilities of its
    // last block have been downloaded
    cudaStreamWaitEvent(p->compute, s.uploaded, 0);
    if (s.used) cudaStreamWaitEvent(p->compute, s.downloaded, 0);
    if (!p->tuned)
    {
        const int err = plan_tune(p, k);
        if (err) return err;
    }
    if (p->use_graph && !s.exec) plan_capture(p, k);
    int err = 0;
    if (s.exec)
    {
        if (cudaGraphLaunch(s.exec, p->compute) != cudaSuccess)
        {
            set_last_error("oskb_tc_plan_enqueue graph",
                    cudaGetLastError());
            return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        }
        ++p->graph_launches;
        for (size_t g = 0; g < s.groups.size(); ++g)
        {
            const size_t off = (size_t) s.groups[g].first * p->problem_bytes;
            cudaStreamWaitEvent(p->out, s.group_events[g], 0);
            if (cudaMemcpyAsync(reinterpret_cast<char*>(vis_host) + off,
                    static_cast<const char*>(s.vis) + off,
                    (size_t) s.groups[g].second * p->problem_bytes,
                    cudaMemcpyDeviceToHost, p->out) != cudaSuccess)
                p->failed = true;
        }
    }
    else
    {
        PlanHook hook{p, k, vis_host};
        p->next_event = 0;
        err = plan_correlate(p, k, p->form, plan_after_group, &hook);
    }
    cudaEventRecord(s.computed, p->compute);
    cudaEventRecord(s.downloaded, p->out);
    s.used = true;
    if (err) return err;
    return p->failed ? OSKB_ERR_MEMORY_COPY_FAILURE : 0;
}

int oskb_tc_plan_wait(oskb_TcPlan* p)
{
    const cudaError_t a = cudaStreamSynchronize(p->in);
    const cudaError_t b = cudaStreamSynchronize(p->compute);
    const cudaError_t c = cudaStreamSynchronize(p->out);
    if (a != cudaSuccess || b != cudaSuccess || c != cudaSuccess ||
            p->failed)
    {
        set_last_error("oskb_tc_plan_wait", cudaGetLastError());
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    return 0;
}

int oskb_tc_plan_form(const oskb_TcPlan* p)
{
    return p ? p->form : 0;
}

int oskb_tc_plan_graph_launches(const oskb_TcPlan* p)
{
    return p ? p->graph_launches : 0;
}

int oskb_tc_plan_tuning_ms(const oskb_TcPlan* p, double* ms)
{
    if (!p || !ms) return OSKB_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < 3; ++i) ms[i] = p->tune_ms[i];
    return 0;
}

}  // extern "C"
