/*
 * bt.h — C ABI of the B200 (sm_100a) bundling library.
 *
 * Drop-in boundary for lpstankus/bundling_thingy's GPU bundling path: the
 * `Gpu` type of the reference binary (src/gpu.rs), its graph loader
 * (src/graph.rs) and the CPU readers of its GPU geometry (src/geometry.rs,
 * src/distortion.rs). Plain pointers and sizes only; no CUDA or torch types.
 *
 * Conventions (mirroring the reference):
 *  - Every call returns a bt_status; 0 is success. On failure a message is
 *    available from bt_last_error(ctx) (ctx may be NULL for calls that fail
 *    before a context exists). This replaces color_eyre::Result.
 *  - A bt_ctx owns all device buffers of one graph (the reference's `Gpu`
 *    owns its buffers and a new upload releases the previous graph,
 *    src/gpu.rs:493-497). All calls on one context are serialised on that
 *    context's CUDA stream; a context must not be used from two threads at
 *    once. Different contexts are independent.
 *  - Host buffers are owned by the caller; the library copies in and out.
 *  - Blocking calls wait for the device with a deadline (60 s by default, as
 *    `Gpu::wait`, src/gpu.rs:484-490; bt_options.wait_seconds changes it)
 *    and return BT_ERR_TIMEOUT past it, leaving the queued work to finish.
 */
#ifndef BT_H
#define BT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BT_ABI_VERSION 3

typedef int32_t bt_status;
enum {
    BT_OK = 0,
    BT_ERR_CAPACITY = 1,       /* resampling exceeds sample capacity (resampling.wgsl overflow 1) */
    BT_ERR_MISMATCH = 2,       /* count and emit passes disagree (resampling.wgsl overflow 2) */
    BT_ERR_INVALID = 3,        /* invalid argument or input data */
    BT_ERR_NO_GRAPH = 4,       /* no uploaded graph ("no uploaded graph", gpu.rs:440) */
    BT_ERR_BUDGET = 5,         /* memory budget exhausted or device allocation failed */
    BT_ERR_TIMEOUT = 6,        /* device wait deadline passed */
    BT_ERR_CUDA = 7,           /* CUDA runtime error */
    BT_ERR_NOT_CONFIGURED = 8, /* "neighbor radius is not configured" (gpu.rs:529-532) */
    BT_ERR_CANCELLED = 9       /* a served request cancelled before admission (bt_server_cancel) */
};

enum { BT_COLOR_BY_DENSITY = 0, BT_COLOR_BY_EDGE_ID = 1 };
/* --palette (src/palette.rs:13-23); 0 is the reference default. */
enum { BT_PALETTE_VIRIDIS = 0, BT_PALETTE_CIVIDIS = 1, BT_PALETTE_PLASMA = 2, BT_PALETTE_BATLOW = 3 };

/* Options of Gpu::new (src/main.rs:34-90, src/gpu.rs:60-168). */
typedef struct bt_options {
    uint32_t width;                 /* map width in texels (headless reference: 1600, gpu.rs:21) */
    uint32_t height;                /* map height in texels */
    uint32_t neighbor_radius;       /* --neighbor-radius in texels; 0 = not configured */
    uint32_t color_by;              /* --color-by; density enables the splat + blur passes */
    uint64_t max_graph_memory_bytes;/* --max-graph-memory-mib * 2^20 (default 1024 MiB) */
    uint32_t evaluate_distortion;   /* --evaluate-distortion: reserves staging bytes, keeps the baseline */
    int32_t device;                 /* CUDA device ordinal */
    /* Extensions beyond the reference (0 selects the reference behaviour): */
    float sample_spacing;           /* resample spacing as a fraction of the canvas; 0 = one texel */
    float blur_sigma;               /* Gaussian sigma in texels; 0 = the fixed sigma-6 table */
    float blur_shrink;              /* sigma factor per density pass; 0 or 1 = none */
    uint32_t fine_cells;            /* neighbour-search cells per grid cell along y (and along x when
                                       fine_cells_x is 0); 0 = automatic */
    uint32_t use_graphs;            /* capture the iteration in a CUDA graph (1 = on, default) */
    uint32_t timing;                /* record per-stage CUDA-event timings */
    uint32_t record_neighbors;      /* keep |N(p)| of the last iteration for bt_read_neighbors */
    uint32_t search_mode;           /* 0: interior search cells from prefix sums, boundary tested
                                       sample by sample; 1: every candidate tested (same results) */
    uint32_t fine_cells_x;          /* neighbour-search cells per grid cell along x; 0 = fine_cells */
    /* Render options of the reference (src/main.rs:59-82), used by bt_render: */
    uint32_t palette;               /* --palette: BT_PALETTE_* */
    uint32_t msaa;                  /* --msaa: 2 or 4 samples per pixel (1 also accepted); 0 = 4 */
    uint32_t endpoint_dots;         /* --endpoint-dots: dots at the first and last sample of each path */
    /* Density-gradient advection, an iteration mode beyond the reference
       (kernel-density-estimation bundling; 0 = the neighbour mean): */
    float advect_step;              /* texels per iteration up the density gradient; > 0 selects the mode
                                       (neighbor_radius must then be 0; density is always accumulated) */
    float advect_smooth;            /* Laplacian relaxation towards the path neighbours, in [0, 1] */
    /* Host deadline of every blocking call on the context, in seconds; past it
       the call returns BT_ERR_TIMEOUT and the work stays queued on the
       device (a later bt_synchronize can still wait for it). 0 = 60 s, the
       reference's Gpu::wait (src/gpu.rs:484-490). */
    float wait_seconds;
    /* 1: bt_iterate and bt_iterate_timed re-check the search-cell shape during
       a job (see bt_iterate); 0 (default): the shape chosen at upload stays. */
    uint32_t shape_checks;
} bt_options;

typedef struct bt_info {
    uint32_t samples;         /* resampled points (Gpu::upload's return, gpu.rs:524) */
    uint32_t paths;           /* edges in the uploaded graph */
    uint32_t drawn_paths;     /* edges with at least two samples */
    uint32_t segments;        /* samples - drawn_paths */
    uint32_t capacity;        /* sample capacity from the budget (resampling.rs:363-370) */
    uint32_t iterations;      /* neighbour-mean iterations since upload */
    uint32_t grid_width;      /* neighbour grid cells (neighbor_mean.rs:26-32) */
    uint32_t grid_height;
    uint32_t fine_cells;      /* search cells per grid cell along y */
    uint32_t density_passes;  /* blur passes since upload */
    uint64_t device_bytes;    /* device memory held by the context */
    uint64_t reserved_bytes;  /* budget accounting of the reference (resampling.rs:394-395) */
    uint32_t fine_cells_x;    /* search cells per grid cell along x */
    uint32_t reserved0;
} bt_info;

typedef struct bt_ctx bt_ctx;
typedef struct bt_graph bt_graph;

/* Library ABI version (BT_ABI_VERSION). */
int32_t bt_abi_version(void);

/* Fills the reference defaults: 1600x1600, density colouring, 1024 MiB. */
void bt_options_init(bt_options* options);

/* Gpu::new (src/gpu.rs:60-168). Validates the options like Resampler::new and
 * GridBuffers::new (src/resampling.rs:72-96, src/neighbor_mean.rs:63-85). */
bt_status bt_create(const bt_options* options, bt_ctx** out);

/* Drop (releases the device buffers and the stream). NULL is ignored. */
void bt_destroy(bt_ctx* ctx);

/* Message of the last failure on ctx, or of the calling thread when ctx is NULL. */
const char* bt_last_error(const bt_ctx* ctx);

/* Gpu::upload (src/gpu.rs:493-525): resample the polylines into evenly spaced
 * samples (resampling.wgsl count_paths/emit_paths), splat and blur the density
 * (density.rs:150-166), and build the neighbour grid for the next iteration.
 * xy holds 2*n_points floats; starts holds n_starts = edges + 1 offsets with
 * starts[0] = 0 and starts[n_starts-1] = n_points (src/graph.rs:7-12). */
bt_status bt_upload(bt_ctx* ctx, const float* xy, uint32_t n_points, const uint32_t* starts,
                    uint32_t n_starts, uint32_t* out_samples);

/* Upload of a parsed graph (Gpu::upload(&Graph)). */
bt_status bt_upload_graph(bt_ctx* ctx, const bt_graph* graph, uint32_t* out_samples);

/* Gpu::iterate (src/gpu.rs:527-553), n times: neighbour mean fused with the
 * density splat, grid rebuild, blur and normalisation (or, with advect_step,
 * one density-gradient advection step fused with the splat, then blur and
 * normalisation). Returns after the work has finished on the device.
 * With options.shape_checks (and search cells not fixed by fine_cells,
 * fine_cells_x), it checks the search-cell shape after 5, 10, 20, 40, ...
 * iterations of an upload: a sampled count of the search's rows and boundary
 * samples, one host wait, and a re-binning when a cost model predicts a
 * saving of more than 8%. Results do not depend on the shape. */
bt_status bt_iterate(bt_ctx* ctx, uint32_t n);

/* Enqueue n iterations without waiting (bt_synchronize waits). Makes no
 * search-shape checks (they wait on the host). */
bt_status bt_iterate_async(bt_ctx* ctx, uint32_t n);
bt_status bt_synchronize(bt_ctx* ctx);

/* bt_iterate, also returning the device milliseconds between CUDA events
 * recorded on the context's stream before and after the n iterations (the
 * reference logs per-pass gpu_ms, src/profiling.rs:127-133); the search-shape
 * checks that fall due are inside that span. */
bt_status bt_iterate_timed(bt_ctx* ctx, uint32_t n, float* device_ms);

bt_status bt_get_info(bt_ctx* ctx, bt_info* info);

/* Changes the context's host deadline (bt_options.wait_seconds; 0 = 60 s) for
 * the blocking calls that follow: the poll loop of Gpu::wait, whose limit the
 * reference fixes at 60 s (src/gpu.rs:484-490). */
bt_status bt_set_wait_seconds(bt_ctx* ctx, float seconds);

/* 12-byte little-endian {f32 x, f32 y, u32 edge_id} records, sample order
 * (the point buffer read by distortion_snapshot, src/gpu.rs:469-482). */
bt_status bt_read_points(bt_ctx* ctx, void* dst, size_t bytes);
/* Checkpoint/resume (beyond the reference, whose bundling state is the point
 * buffer that distortion_snapshot reads, src/gpu.rs:469-482): bt_read_points
 * gives the checkpoint; this puts its positions back into the uploaded graph
 * (the same graph and options, after bt_upload) as the state after
 * `iterations` iterations: the positions are re-binned for the next
 * iteration and their density recomputed with that iteration's density pass,
 * so iterating on gives the same results as an uninterrupted run. Records
 * whose edge ids differ from the uploaded graph's, or whose positions are
 * not finite, are refused with BT_ERR_INVALID. */
bt_status bt_restore_points(bt_ctx* ctx, const void* records, size_t bytes, uint32_t iterations);
/* 12-byte {u32 point_offset, u32 segment_offset, u32 count} per edge
 * (distortion_layout, src/gpu.rs:438-467). Skipped edges read as zeros. */
bt_status bt_read_paths(bt_ctx* ctx, void* dst, size_t bytes);
/* Segment start indices (resampling.wgsl segments buffer), samples - drawn_paths entries. */
bt_status bt_read_segments(bt_ctx* ctx, uint32_t* dst, size_t count);
/* Edge endpoints {x0, y0, x1, y1} per edge (resampling.wgsl edges buffer). */
bt_status bt_read_edges(bt_ctx* ctx, float* dst, size_t count);
/* Normalised density, width*height f32 in [0,1] (normalization.wgsl; the
 * reference stores it in the R channel of an RGBA16F texture). */
bt_status bt_read_density(bt_ctx* ctx, float* dst, size_t count);
/* Blurred density before normalisation and its maximum (blur.wgsl outputs). */
bt_status bt_read_density_raw(bt_ctx* ctx, float* dst, size_t count, float* peak);
/* Splat counts of the last density pass, width*height u32. */
bt_status bt_read_counts(bt_ctx* ctx, uint32_t* dst, size_t count);
/* Neighbour-grid cell ids (spatial_grid.wgsl:67-70) of the current samples,
 * sample order. Requires a configured radius. */
bt_status bt_read_cells(bt_ctx* ctx, uint32_t* dst, size_t count);
/* No counterpart in the reference. Work of the next iteration's neighbour
 * search under the current search cells, over every `stride`-th slot (1 =
 * all): search rows, samples in boundary cells (tested one by one; the
 * interior cells come from prefix sums) and movable samples counted. The
 * search-shape checks of bt_iterate use the same count. */
bt_status bt_search_stats(bt_ctx* ctx, uint32_t stride, uint64_t* rows, uint64_t* boundary, uint64_t* probed);
/* The grid binning that the next iteration will search: samples listed by
 * search cell (slot order, `count` = samples) and the start slot of each
 * search cell (cell_count = fine grid cells + 1). */
bt_status bt_read_binning(bt_ctx* ctx, uint32_t* slot_samples, size_t count, uint32_t* cell_starts,
                          size_t cell_count);
/* Neighbour count |N(p)| of every sample in the last iteration (0 for
 * endpoints), sample order. */
bt_status bt_read_neighbors(bt_ctx* ctx, uint32_t* dst, size_t count);

/* Distortion of the current geometry against the geometry at upload
 * (src/main.rs:159-180, src/distortion.rs:172-216); requires
 * evaluate_distortion. size is the canvas size in pixels (gpu::SIZE). */
bt_status bt_distortion(bt_ctx* ctx, uint32_t size, double* distortion, double* rms_displacement_pixels);

/* Gpu::render + Gpu::readback (src/gpu.rs:572-655) of the headless export:
 * rasterises the current paths (and the endpoint dots when endpoint_dots is
 * set) into width x height RGBA8 pixels, rows from the top, with the options'
 * palette, colouring and msaa; before any upload, the blank frame (the clear
 * colour) the noisiness report calibrates its background on
 * (src/main.rs:115-121). rgba (rgba_bytes = 4*width*height) may be NULL;
 * colored_pixels (may be NULL) receives the number of pixels whose RGB
 * differs from the clear colour (noisiness::measure, src/noisiness.rs:44-56);
 * device_ms (may be NULL) the device time of the frame's kernels. The
 * rasterisation rules are stated in csrc/render.cu; agreement with a
 * hardware rasteriser is approximate. */
bt_status bt_render(bt_ctx* ctx, uint8_t* rgba, size_t rgba_bytes, uint64_t* colored_pixels, float* device_ms);

/* Per-stage device milliseconds of the last upload/iteration, as the
 * reference's GpuTimings (src/profiling.rs:35-136). names/ms hold `capacity`
 * entries; returns the number of stages in *count. */
bt_status bt_stage_times(bt_ctx* ctx, const char** names, float* ms, uint32_t capacity, uint32_t* count);

/* Autotuner (beyond the reference): times `iterations` iterations of this
 * graph (after one warm-up iteration, CUDA events on the context's stream)
 * for each candidate search-cell shape — rows of 4, 2, 1 and 1/2 texels
 * (fine_cells = r/4, r/2, r, 2r) with cells 1, 2 or 4 times narrower than
 * high (fine_cells_x), at most 32 Mi search cells — and writes the fastest
 * options to *tuned (its time to *best_ms when not NULL). Every candidate
 * gives bit-identical results. */
bt_status bt_autotune(const bt_options* options, const float* xy, uint32_t n_points, const uint32_t* starts,
                      uint32_t n_starts, uint32_t iterations, bt_options* tuned, float* best_ms);

/* ---- Batches: many independent graphs per launch ----
 *
 * Beyond the reference (which bundles one graph at a time, src/main.rs:113-126):
 * each graph occupies a slot with its own options (map size, radius, sigma,
 * spacing); bt_batch_iterate advances every active slot by n iterations of
 * Gpu::iterate with one set of persistent launches over a graph x tile work
 * queue, captured in a CUDA graph. A slot's results equal a bt_ctx run of the
 * same graph bit for bit, whatever else is in the batch. */
typedef struct bt_batch bt_batch;

bt_status bt_batch_create(int32_t device, bt_batch** out);
void bt_batch_destroy(bt_batch* batch);
const char* bt_batch_last_error(const bt_batch* batch);
/* Uploads one graph (bt_create + bt_upload with `options`; neighbor_radius
 * must be set) into a free slot; returns its slot index and sample count. */
bt_status bt_batch_add(bt_batch* batch, const bt_options* options, const float* xy, uint32_t n_points,
                       const uint32_t* starts, uint32_t n_starts, uint32_t* slot, uint32_t* samples);
/* Uploads `count` graphs at once (arrays of per-graph arguments as in
 * bt_batch_add): every graph's upload runs on its own stream with two host
 * waits in total. All or nothing: on failure no slot is added. */
bt_status bt_batch_add_many(bt_batch* batch, uint32_t count, const bt_options* options, const float* const* xy,
                            const uint32_t* n_points, const uint32_t* const* starts, const uint32_t* n_starts,
                            uint32_t* slots, uint32_t* samples);
/* Releases a slot (its index may be reused by a later add). */
bt_status bt_batch_remove(bt_batch* batch, uint32_t slot);
/* n iterations of every active slot; waits for the device. */
bt_status bt_batch_iterate(bt_batch* batch, uint32_t n);
bt_status bt_batch_iterate_async(bt_batch* batch, uint32_t n);
bt_status bt_batch_synchronize(bt_batch* batch);
/* bt_batch_iterate with the device milliseconds of the n iterations. */
bt_status bt_batch_iterate_timed(bt_batch* batch, uint32_t n, float* device_ms);
bt_status bt_batch_slot_count(bt_batch* batch, uint32_t* active, uint32_t* capacity);
/* Slots of at least `samples` samples iterate on their own context's stream
 * and CUDA graphs, beside the persistent step and concurrently with it,
 * instead of joining its work lists (0 or UINT32_MAX = every slot joins, the
 * default). Large dense graphs run faster that way; mid-size graphs on small
 * maps run faster in the step. Applies to every slot from the next
 * iteration; results are the same either way. */
bt_status bt_batch_set_solo_samples(bt_batch* batch, uint32_t samples);
/* Work shape of the batch's neighbour-mean step (the reference's counterpart
 * knob is the compute workgroup size of its kernels, src/neighbor_mean.rs:4,
 * src/resampling.rs:19): samples per mean tile, which is also the CTA size
 * (64, 128 or 256; default 128), and resident mean CTAs per SM (0 = as many
 * as fit, the default). Results do not depend on it; from the next step. */
bt_status bt_batch_set_shape(bt_batch* batch, uint32_t mean_tile, uint32_t mean_ctas_per_sm);
bt_status bt_batch_get_shape(bt_batch* batch, uint32_t* mean_tile, uint32_t* mean_ctas_per_sm);
/* Autotuner of the batch shape (beyond the reference): uploads the graphs
 * (arguments as bt_batch_add_many) into a scratch batch for each candidate
 * shape, times `iterations` iterations after the upload (CUDA events) and
 * returns the fastest shape (its time to *best_ms when not NULL). The
 * caller's own batches are not touched; pass the result to
 * bt_batch_set_shape. */
bt_status bt_batch_autotune(int32_t device, uint32_t count, const bt_options* options, const float* const* xy,
                            const uint32_t* n_points, const uint32_t* const* starts, const uint32_t* n_starts,
                            uint32_t iterations, uint32_t* mean_tile, uint32_t* mean_ctas_per_sm, float* best_ms);
/* The context of a slot, for the bt_read_* and bt_get_info calls; owned by
 * the batch (do not destroy or iterate it). Waits for the batch's work. */
bt_ctx* bt_batch_slot(bt_batch* batch, uint32_t slot);

/* ---- Serving: continuous batching of arriving requests ----
 *
 * Beyond the reference (its CLI bundles one graph per process run,
 * src/main.rs:113-126). A worker thread owns one bt_batch. Submitted requests
 * become visible at their arrival time; the worker admits them in arrival
 * order while the device-memory budget and `max_active` allow, uploads every
 * admitted graph concurrently on its own stream while the batch iterates,
 * joins them to the batch between iterations, and takes each graph out of the
 * batch the moment its own iteration count is reached. Admission generalises
 * Allocation::new (src/resampling.rs:321-397) from one graph to all resident
 * graphs: every device allocation any request makes is charged against
 * `budget_bytes` before it is made; a request that does not fit waits (idle
 * pooled contexts are freed first) until resident graphs finish or results
 * are released, and fails with BT_ERR_BUDGET only when it does not fit alone.
 * Results stay on the device until read and released, and equal a standalone
 * bt_ctx run of the same graph bit for bit. All calls are thread-safe. */
typedef struct bt_server bt_server;

typedef struct bt_server_options {
    int32_t device;
    uint32_t max_active;      /* graphs uploading or iterating at once (0 = unlimited) */
    uint64_t budget_bytes;    /* device memory of all resident graphs and pooled contexts */
    uint32_t max_step;        /* batch iterations between admission points while requests wait to join (>= 1) */
    uint32_t solo_samples;    /* requests of at least this many samples fill the device alone: they iterate
                                 on their own context's stream and CUDA graphs beside the batch instead of
                                 joining it (0 = 32768; UINT32_MAX = every request joins the batch) */
    uint64_t reserve_bytes;   /* device memory mapped into the allocator's pool at creation, so that
                                 admissions do not map memory while steps run (0 = none; at most
                                 budget_bytes) */
    uint32_t queue_timeout_ms;/* a request still waiting for admission this long after its arrival
                                 fails with BT_ERR_TIMEOUT (0 = it waits as long as it takes) */
    uint32_t reserved[3];
} bt_server_options;

typedef struct bt_request_result {
    uint64_t id;
    int32_t status;           /* BT_OK, or why the request failed */
    uint32_t samples;
    uint32_t iterations;
    uint32_t reserved0;
    double arrival_s;         /* server clock (seconds since bt_server_create) */
    double admitted_s;        /* upload started */
    double finished_s;        /* results ready on the device, batch slot freed */
    uint64_t device_bytes;    /* device memory the request's graph held */
    char message[160];
} bt_request_result;

typedef struct bt_server_stats {
    uint64_t submitted, finished, failed;
    uint64_t steps, rebuilds, budget_waits, evictions;
    uint32_t queued, active, peak_active, resident_results;
    uint64_t device_bytes, peak_device_bytes;
    /* Seconds the worker spent launching batch steps (with rebuilds),
     * uploading (admission and upload phases), waiting for steps, retiring
     * and publishing finished graphs, and idle. */
    double launch_s, upload_s, wait_s, retire_s, idle_s;
    uint64_t contexts_created;   /* device contexts made (the rest were reused) */
    double create_s;             /* of upload_s: seconds spent making contexts */
} bt_server_stats;

/* device 0, max_active 32, budget 120 GB (120e9 bytes), max_step 1, no reserve. */
void bt_server_options_init(bt_server_options* options);
bt_status bt_server_create(const bt_server_options* options, bt_server** out);
/* Stops the worker; unfinished requests are dropped. */
void bt_server_destroy(bt_server* server);
const char* bt_server_last_error(const bt_server* server);
/* Seconds since bt_server_create (the clock of arrival and result times). */
double bt_server_clock(const bt_server* server);
/* Copies the graph and queues it: `iterations` bt_iterate steps with
 * `options` (neighbor_radius must be set). The request arrives at
 * `arrival_s` on the server clock (a negative value = now; a future time
 * replays a recorded arrival schedule). */
bt_status bt_server_submit(bt_server* server, const bt_options* options, const float* xy, uint32_t n_points,
                           const uint32_t* starts, uint32_t n_starts, uint32_t iterations, double arrival_s,
                           uint64_t* id);
/* The next request to finish or fail that was not returned before, in
 * completion order; waits up to timeout_s (BT_ERR_TIMEOUT if none). */
bt_status bt_server_next(bt_server* server, double timeout_s, bt_request_result* result);
/* 12-byte {x, y, edge_id} records of a finished request, as bt_read_points. */
bt_status bt_server_read_points(bt_server* server, uint64_t id, void* dst, size_t bytes);
/* The finished request's context, for the other bt_read_* and bt_get_info
 * calls until it is released; owned by the server (do not destroy or iterate
 * it). NULL if the request has not finished or failed. */
bt_ctx* bt_server_result(bt_server* server, uint64_t id);
/* Gives a finished or failed request's memory back to the server. */
bt_status bt_server_release(bt_server* server, uint64_t id);
/* Asks the server to drop a request that is still queued (not yet
 * admitted): it then finishes with BT_ERR_CANCELLED through bt_server_next
 * and holds no device memory. A request already admitted runs to the end and
 * reports its own status. BT_ERR_INVALID for an unknown or finished id. */
bt_status bt_server_cancel(bt_server* server, uint64_t id);
bt_status bt_server_stats_get(bt_server* server, bt_server_stats* stats);

/* ---- Density blur without allocation ---- */

/* Largest width*height accepted by bt_density_noalloc: its static device
 * scratch holds one f32 image of this many texels (4 MiB) plus a 256-byte
 * head, on every GPU that loads the library, until the process exits. */
#define BT_NOALLOC_MAX_TEXELS (1024u * 1024u)

/* No counterpart in the reference. The density blur and normalisation
 * (the same kernels and results as the density passes of bt_upload and
 * bt_iterate) for callers that may not allocate device memory: a plugin or
 * renderer whose host application owns every device allocation, or a frame
 * loop that cannot take cudaMalloc's implicit device synchronisation or an
 * allocation failure mid-frame. The caller passes device pointers to
 * width*height u32 splat counts (4-byte aligned) and to the width*height f32
 * output (16-byte aligned: it is written four texels at a time); misaligned
 * buffers are rejected with BT_ERR_INVALID before anything is launched. A
 * cudaStream_t goes in `stream` (NULL = the default stream); the call is
 * asynchronous on that stream. It calls no cudaMalloc or cudaFree: its one
 * intermediate image lives in a file-scope static device array of
 * BT_NOALLOC_MAX_TEXELS texels, and larger maps are rejected with
 * BT_ERR_INVALID. The first call on a device performs a one-time set-up on
 * the current device (the array's device address and the kernels'
 * shared-memory attribute); make that first call before any stream capture.
 * A set-up that fails returns BT_ERR_CUDA and is tried again by the next call.
 * Every call shares the one array per device, so calls whose work overlaps on
 * the GPU race: serialise them (one stream, or events between streams).
 * blur_sigma as bt_options.blur_sigma (0 = the fixed sigma-6 table). */
bt_status bt_density_noalloc(const uint32_t* counts, float* density, uint32_t width, uint32_t height,
                             float blur_sigma, void* stream);

/* ---- Graph loader (src/graph.rs) ---- */

/* Graph::parse (src/graph.rs:35-77). */
bt_status bt_graph_parse(const char* text, size_t len, bt_graph** out);
/* Graph::load (src/graph.rs:22-33). */
bt_status bt_graph_load(const char* path, bt_graph** out);
void bt_graph_free(bt_graph* graph);
uint32_t bt_graph_point_count(const bt_graph* graph);
uint32_t bt_graph_start_count(const bt_graph* graph);
const float* bt_graph_points(const bt_graph* graph);      /* Graph::points, 2 floats per point */
const uint32_t* bt_graph_starts(const bt_graph* graph);   /* Graph::starts */
/* Graph::normalization (src/graph.rs:79-91): {min_x, min_y, scale, tx, ty}. */
bt_status bt_graph_normalization(const bt_graph* graph, float out[5]);

/* ---- CPU readers of GPU geometry (src/geometry.rs, src/distortion.rs) ---- */

/* Layout::new (src/geometry.rs:28-73): checks that path reservations tile
 * [0, samples) and segments tile [0, samples - edges). paths holds 3 u32 per
 * edge. Returns BT_ERR_INVALID with the reference's message otherwise. */
bt_status bt_layout_check(const uint32_t* paths, uint32_t n_paths, uint32_t samples);
/* Decoder::push/finish (src/geometry.rs:131-187): decodes 12-byte records to
 * 2 floats per sample, checking edge ids and finiteness. */
bt_status bt_decode_points(const uint32_t* paths, uint32_t n_paths, uint32_t samples, const void* records,
                           size_t bytes, float* xy);
/* squared_integral (src/distortion.rs:137-168) of two f32 curves. */
bt_status bt_squared_integral(const float* original, size_t n_original, const float* current,
                              size_t n_current, double* out);

#ifdef __cplusplus
}
#endif

#endif /* BT_H */
