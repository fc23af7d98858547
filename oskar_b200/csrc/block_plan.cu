// Block plan: the host driver for the direct block correlator.
//
// Owns, for one block shape (stations, sources, dumps, channels, source and
// smearing kinds), the device copies of the sky, station offsets and beam,
// the per-block device inputs (station uvw per dump, hour angle per dump),
// the device visibility block, and page-locked host buffers for what
// changes from block to block. One block is
//     H2D uvw and hour angles -> clear visibilities -> correlate (one
//     persistent launch) -> D2H visibilities
// on the plan's own stream. The first execute runs the sequence eagerly
// (the correlator picks its launch schedule then) and captures it into a
// CUDA graph; every later execute replays that graph, so a block costs one
// graph launch on the host. This is the B200 form of the reference's
// per-block loop over (dump, chunk, channel) in sim_baselines
// (oskar/interferometer/src/oskar_interferometer_run_block.c:156-336), whose
// visibility block is cleared per block (run_block.c:55) and copied to the
// host for finalisation (oskar_interferometer_finalise_block.c:32-40).
// With a spectral sky the plan scales every source's brightness to every
// channel once, when the sky is set, instead of once per (dump, channel) as
// the reference's block loop does (run_block.c:183-190).
#include <stdlib.h>
#include <string.h>

#include "common.cuh"

struct oskb_BlockPlan
{
    int elem;  // 8: double, 4: float
    int casa, num_st, num_src, num_times, num_channels;
    int gaussian, with_beam, beam_per_dump;
    double bandwidth_hz, time_avg_sec, dec0_rad;
    double uv_min, uv_max, filter_min, filter_max;
    int uv_units;
    // device
    void* sky[10];  // I, Q, U, V, l, m, n, a, b, c
    void *st_x, *st_y, *E, *uvw, *vis;
    double *inv_wl, *gha0, *freq;
    // Spectral sky: brightness per channel [channel][source] (4 arrays),
    // scaled once from the sky table when it is set.
    void* flux_c[4];
    // host (page-locked)
    void *h_uvw, *h_vis;
    double* h_gha0;
    size_t uvw_bytes, vis_bytes, e_bytes;
    cudaStream_t stream;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int graph_launches;
};

namespace {

int enqueue_block(oskb_BlockPlan* p)
{
    cudaStream_t s = p->stream;
    if (cudaMemcpyAsync(p->uvw, p->h_uvw, p->uvw_bytes,
            cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(p->gha0, p->h_gha0, sizeof(double) *
            p->num_times, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemsetAsync(p->vis, 0, p->vis_bytes, s) != cudaSuccess)
    {
        oskb::set_last_error("block plan", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    int err;
    void* const* k = p->sky;
    void* const* f = p->flux_c[0] ? p->flux_c : p->sky;
    const long long fs = p->flux_c[0] ? p->num_src : 0;
    if (p->elem == 8)
        err = oskb_correlate_block_direct_spectral_d(p->casa, p->num_src,
                p->num_st, p->num_times, p->num_channels,
                (const double*) p->E, p->beam_per_dump, (const double*) f[0],
                (const double*) f[1], (const double*) f[2],
                (const double*) f[3], fs,
                (const double*) k[4], (const double*) k[5],
                (const double*) k[6], (const double*) k[7],
                (const double*) k[8], (const double*) k[9],
                (const double*) p->uvw, (const double*) p->st_x,
                (const double*) p->st_y, p->inv_wl, p->bandwidth_hz,
                p->time_avg_sec, p->gha0, p->dec0_rad, p->uv_min, p->uv_max,
                p->uv_units, p->filter_min, p->filter_max,
                (double*) p->vis, s);
    else
        err = oskb_correlate_block_direct_spectral_f(p->casa, p->num_src,
                p->num_st, p->num_times, p->num_channels,
                (const float*) p->E, p->beam_per_dump, (const float*) f[0],
                (const float*) f[1], (const float*) f[2],
                (const float*) f[3], fs,
                (const float*) k[4], (const float*) k[5],
                (const float*) k[6], (const float*) k[7],
                (const float*) k[8], (const float*) k[9],
                (const float*) p->uvw, (const float*) p->st_x,
                (const float*) p->st_y, p->inv_wl, p->bandwidth_hz,
                p->time_avg_sec, p->gha0, p->dec0_rad, p->uv_min, p->uv_max,
                p->uv_units, p->filter_min, p->filter_max,
                (float*) p->vis, s);
    if (err) return err;
    if (cudaMemcpyAsync(p->h_vis, p->vis, p->vis_bytes,
            cudaMemcpyDeviceToHost, s) != cudaSuccess)
    {
        oskb::set_last_error("block plan", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}

int upload(void* dst, const void* src, size_t bytes)
{
    if (!src || !dst) return OSKB_ERR_INVALID_ARGUMENT;
    if (cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    {
        oskb::set_last_error("block plan upload", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}

}  // namespace

extern "C" {

void oskb_block_plan_free(oskb_BlockPlan* p)
{
    if (!p) return;
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (int i = 0; i < 10; ++i) cudaFree(p->sky[i]);
    for (int i = 0; i < 4; ++i) cudaFree(p->flux_c[i]);
    cudaFree(p->st_x); cudaFree(p->st_y); cudaFree(p->E); cudaFree(p->uvw);
    cudaFree(p->vis); cudaFree(p->inv_wl); cudaFree(p->gha0);
    cudaFree(p->freq);
    cudaFreeHost(p->h_uvw); cudaFreeHost(p->h_vis); cudaFreeHost(p->h_gha0);
    if (p->stream) cudaStreamDestroy(p->stream);
    free(p);
}

oskb_BlockPlan* oskb_block_plan_create(int precision_bytes, int casa,
        int num_stations, int num_sources, int num_times, int num_channels,
        int gaussian, int with_beam, int beam_per_dump,
        const double* frequency_hz, double channel_bandwidth_hz,
        double time_average_sec, double dec0_rad, double uv_min,
        double uv_max, int uv_filter_units, double source_filter_min,
        double source_filter_max, int* status)
{
    if (*status) return nullptr;
    if ((precision_bytes != 8 && precision_bytes != 4) || num_stations < 2 ||
            num_sources < 1 || num_times < 1 || num_channels < 1 ||
            !frequency_hz)
    {
        *status = OSKB_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    oskb_BlockPlan* p = (oskb_BlockPlan*) calloc(1, sizeof(oskb_BlockPlan));
    p->elem = precision_bytes;
    p->casa = casa; p->num_st = num_stations; p->num_src = num_sources;
    p->num_times = num_times; p->num_channels = num_channels;
    p->gaussian = gaussian; p->with_beam = with_beam;
    p->beam_per_dump = beam_per_dump;
    p->bandwidth_hz = channel_bandwidth_hz;
    p->time_avg_sec = time_average_sec; p->dec0_rad = dec0_rad;
    p->uv_min = uv_min; p->uv_max = uv_max; p->uv_units = uv_filter_units;
    p->filter_min = source_filter_min; p->filter_max = source_filter_max;
    const size_t e = precision_bytes, ns = num_sources, nst = num_stations;
    const size_t nbl = nst * (nst - 1) / 2;
    p->uvw_bytes = e * 3 * nst * num_times;
    p->vis_bytes = e * 8 * nbl * num_channels * num_times;
    p->e_bytes = with_beam ? e * 8 * nst * ns * (beam_per_dump ? num_times
            : 1) : 0;
    bool ok = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) ==
            cudaSuccess;
    for (int i = 0; i < 10 && ok; ++i)
        if (i < 7 || gaussian) ok = cudaMalloc(&p->sky[i], e * ns) ==
                cudaSuccess && cudaMemset(p->sky[i], 0, e * ns) ==
                cudaSuccess;
    ok = ok && cudaMalloc(&p->st_x, e * nst) == cudaSuccess &&
            cudaMalloc(&p->st_y, e * nst) == cudaSuccess &&
            cudaMalloc(&p->uvw, p->uvw_bytes) == cudaSuccess &&
            cudaMalloc(&p->vis, p->vis_bytes) == cudaSuccess &&
            cudaMalloc((void**) &p->inv_wl, sizeof(double) * num_channels)
            == cudaSuccess &&
            cudaMalloc((void**) &p->gha0, sizeof(double) * num_times) ==
            cudaSuccess &&
            cudaMalloc((void**) &p->freq, sizeof(double) * num_channels) ==
            cudaSuccess &&
            (!with_beam || cudaMalloc(&p->E, p->e_bytes) == cudaSuccess) &&
            cudaMallocHost(&p->h_uvw, p->uvw_bytes) == cudaSuccess &&
            cudaMallocHost(&p->h_vis, p->vis_bytes) == cudaSuccess &&
            cudaMallocHost((void**) &p->h_gha0, sizeof(double) * num_times)
            == cudaSuccess;
    if (ok)
    {
        double* inv = (double*) malloc(sizeof(double) * num_channels);
        for (int c = 0; c < num_channels; ++c)
            inv[c] = frequency_hz[c] / 299792458.0;
        ok = cudaMemcpy(p->inv_wl, inv, sizeof(double) * num_channels,
                cudaMemcpyHostToDevice) == cudaSuccess &&
                cudaMemcpy(p->freq, frequency_hz, sizeof(double) *
                num_channels, cudaMemcpyHostToDevice) == cudaSuccess &&
                cudaMemset(p->st_x, 0, e * nst) == cudaSuccess &&
                cudaMemset(p->st_y, 0, e * nst) == cudaSuccess;
        free(inv);
        memset(p->h_uvw, 0, p->uvw_bytes);
        memset(p->h_gha0, 0, sizeof(double) * num_times);
    }
    if (!ok)
    {
        oskb::set_last_error("oskb_block_plan_create", cudaGetLastError());
        oskb_block_plan_free(p);
        *status = OSKB_ERR_MEMORY_ALLOC_FAILURE;
        return nullptr;
    }
    return p;
}

int oskb_block_plan_set_sky(oskb_BlockPlan* p, const void* I, const void* Q,
        const void* U, const void* V, const void* l, const void* m,
        const void* n, const void* a, const void* b, const void* c)
{
    const void* src[10] = {I, Q, U, V, l, m, n, a, b, c};
    const size_t bytes = (size_t) p->elem * p->num_src;
    for (int i = 0; i < (p->gaussian ? 10 : 7); ++i)
    {
        if (i < 4 && !src[i] && p->flux_c[0]) continue;
        if (int err = upload(p->sky[i], src[i], bytes)) return err;
    }
    return 0;
}

int oskb_block_plan_set_spectral_sky(oskb_BlockPlan* p, int capacity,
        int num_columns, const void* table, const int* num_valid_columns,
        const int* columns)
{
    if (!table || !num_valid_columns || !columns || capacity < p->num_src ||
            num_columns < 1)
        return OSKB_ERR_INVALID_ARGUMENT;
    const size_t e = p->elem, ns = p->num_src;
    const size_t table_bytes = e * (size_t) capacity * num_columns;
    const size_t nv_bytes = sizeof(int) * 20 * ns;
    const size_t flux_bytes = e * ns * p->num_channels;
    void *d_table = nullptr, *d_nv = nullptr;
    bool ok = cudaMalloc(&d_table, table_bytes) == cudaSuccess &&
            cudaMalloc(&d_nv, nv_bytes) == cudaSuccess;
    for (int i = 0; i < 4 && ok; ++i)
        if (!p->flux_c[i])
            ok = cudaMalloc(&p->flux_c[i], flux_bytes) == cudaSuccess;
    int err = ok ? 0 : OSKB_ERR_MEMORY_ALLOC_FAILURE;
    if (ok)
    {
        err = upload(d_table, table, table_bytes);
        if (!err) err = upload(d_nv, num_valid_columns, nv_bytes);
    }
    if (!err)
    {
        if (p->elem == 8)
            err = oskb_sky_scale_flux_channels_d(p->num_src, capacity,
                    num_columns, p->num_channels, p->freq,
                    (const double*) d_table, (const int*) d_nv, columns,
                    p->num_src, (double*) p->flux_c[0],
                    (double*) p->flux_c[1], (double*) p->flux_c[2],
                    (double*) p->flux_c[3], p->stream);
        else
            err = oskb_sky_scale_flux_channels_f(p->num_src, capacity,
                    num_columns, p->num_channels, p->freq,
                    (const float*) d_table, (const int*) d_nv, columns,
                    p->num_src, (float*) p->flux_c[0],
                    (float*) p->flux_c[1], (float*) p->flux_c[2],
                    (float*) p->flux_c[3], p->stream);
    }
    if (cudaStreamSynchronize(p->stream) != cudaSuccess && !err)
        err = OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    cudaFree(d_table);
    cudaFree(d_nv);
    if (err)
    {
        if (!ok) oskb::set_last_error("oskb_block_plan_set_spectral_sky",
                cudaGetLastError());
        for (int i = 0; i < 4; ++i)
        {
            cudaFree(p->flux_c[i]);
            p->flux_c[i] = nullptr;
        }
    }
    // The captured block reads the brightness arrays: capture again.
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->exec = nullptr;
    p->graph = nullptr;
    return err;
}

int oskb_block_plan_set_stations(oskb_BlockPlan* p, const void* ecef_x,
        const void* ecef_y)
{
    const size_t bytes = (size_t) p->elem * p->num_st;
    if (int err = upload(p->st_x, ecef_x, bytes)) return err;
    return upload(p->st_y, ecef_y, bytes);
}

int oskb_block_plan_set_beam(oskb_BlockPlan* p, const void* E)
{
    if (!p->with_beam) return OSKB_ERR_INVALID_ARGUMENT;
    return upload(p->E, E, p->e_bytes);
}

void* oskb_block_plan_host_uvw(oskb_BlockPlan* p) { return p->h_uvw; }
double* oskb_block_plan_host_gha0(oskb_BlockPlan* p) { return p->h_gha0; }
const void* oskb_block_plan_host_vis(oskb_BlockPlan* p) { return p->h_vis; }

int oskb_block_plan_execute(oskb_BlockPlan* p)
{
    if (p->exec)
    {
        if (cudaGraphLaunch(p->exec, p->stream) != cudaSuccess)
        {
            oskb::set_last_error("oskb_block_plan_execute",
                    cudaGetLastError());
            return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
        }
        ++p->graph_launches;
        return 0;
    }
    // First block: eager (fixes the launch schedule), then capture.
    if (int err = enqueue_block(p)) return err;
    if (cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeRelaxed)
            != cudaSuccess)
    {
        oskb::set_last_error("block plan capture", cudaGetLastError());
        return 0;  // the block ran; later blocks run eagerly too
    }
    const int err = enqueue_block(p);
    cudaGraph_t g = nullptr;
    const cudaError_t e1 = cudaStreamEndCapture(p->stream, &g);
    if (err || e1 != cudaSuccess || !g ||
            cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess)
    {
        if (g) cudaGraphDestroy(g);
        p->exec = nullptr;
        cudaGetLastError();
        return 0;
    }
    p->graph = g;
    return 0;
}

int oskb_block_plan_synchronize(oskb_BlockPlan* p)
{
    const cudaError_t e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess)
    {
        oskb::set_last_error("oskb_block_plan_synchronize", e);
        return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
    }
    return 0;
}

int oskb_block_plan_graph_launches(const oskb_BlockPlan* p)
{
    return p->exec ? p->graph_launches : -1;
}

}  // extern "C"
