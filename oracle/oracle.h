/*
 * oracle.h — CPU restatement of lpstankus/bundling_thingy's edge-bundling loop.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links or calls this code;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do, and
 * only as the checker or the timed CPU baseline.
 *
 * PARITY UNPINNED: the reference ships no golden vectors, fixtures or tests
 * (its repository forbids them), its data files are Git-LFS stubs, and it
 * cannot be compiled or run here (Rust + wgpu/Vulkan; no rustc, no graphics
 * stack). This restatement is pinned only against hand-derived known answers
 * (tests/test_oracle_kat.py) and by reading the WGSL/Rust sources it cites.
 *
 * Every float formula is the reference's expression evaluated left to right
 * with IEEE single precision, one rounding per operation (compiled with
 * -ffp-contract=off), except where a comment names a fused multiply-add.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parsed trail graph (src/graph.rs:7-12). xy holds 2*n_points floats. */
typedef struct or_graph {
    float* xy;
    uint32_t n_points;
    uint32_t* starts;   /* n_starts = edges + 1, trailing sentinel */
    uint32_t n_starts;
    float min[2], max[2];
} or_graph;

/* src/graph.rs:35-77. Returns 0 on success, nonzero with a message otherwise. */
int or_parse_trl(const char* text, size_t len, or_graph* out, char* err, size_t errlen);
void or_graph_free(or_graph* g);

/* src/graph.rs:79-91: out = {min_x, min_y, scale, translation_x, translation_y}. */
int or_normalization(const float min[2], const float max[2], float out[5], char* err, size_t errlen);

/* Blur taps for a given sigma (0 = the reference's fixed sigma-6 table,
 * src/shaders/blur.wgsl:42-60). Writes w[0..R] and returns R, or -1. */
int or_blur_weights(double sigma, float* w, int max_taps);

typedef struct or_config {
    uint32_t width, height;     /* map size in texels (src/gpu.rs:99-107) */
    uint32_t radius;            /* neighbour radius in texels; 0 = not configured */
    uint32_t accumulate_density;/* color_by == density (src/resampling.rs:123-126) */
    float resample_scale[2];    /* resampling texel_scale; reference: (size-1)*0.5 */
    uint32_t capacity;          /* sample capacity (src/resampling.rs:363-370) */
    double sigma;               /* blur sigma in texels; 0 = reference fixed table */
    double shrink;              /* sigma factor per density pass; 1 = none */
    int threads;                /* OpenMP threads; 0 = default */
} or_config;

typedef struct or_state or_state;

or_state* or_create(const or_config* cfg);
void or_destroy(or_state* s);
/* Gpu::upload (src/gpu.rs:493-525). status: 0 ok, 1 capacity overflow,
 * 2 count/emit mismatch, 3 invalid input. */
int or_upload(or_state* s, const float* xy, uint32_t n_points, const uint32_t* starts,
              uint32_t n_starts, uint32_t* samples, char* err, size_t errlen);
/* Gpu::iterate (src/gpu.rs:527-553), n times. mode 0 = exact fixed-point
 * accumulation (canonical), 1 = f32 running sum in ascending-index order. */
int or_iterate(or_state* s, uint32_t n, int mode);

uint32_t or_samples(const or_state* s);
uint32_t or_paths(const or_state* s);
void or_get_points(const or_state* s, float* xy, uint32_t* edge_ids);
void or_get_paths(const or_state* s, uint32_t* paths /* 3 per path */);
void or_get_segments(const or_state* s, uint32_t* segments /* samples - edges */);
void or_get_edges(const or_state* s, float* edges /* 4 per path */);
void or_get_counts(const or_state* s, uint32_t* counts);
void or_get_blurred(const or_state* s, float* horizontal, float* vertical, float* peak);
void or_get_normalized(const or_state* s, float* out);
/* Cell ids (src/shaders/spatial_grid.wgsl:59-70) of the current positions. */
void or_get_cells(const or_state* s, uint32_t* cell_ids, uint32_t* grid_w, uint32_t* grid_h);
/* Neighbour counts of the last iteration (n including the point itself). */
void or_get_neighbors(const or_state* s, uint32_t* neighbors);

/* Pure kernels on caller data. */
void or_splat(const float* xy, size_t n, uint32_t w, uint32_t h, uint32_t* counts);
void or_blur(const uint32_t* counts, uint32_t w, uint32_t h, const float* taps, int R,
             float* horizontal, float* vertical, float* peak);
void or_normalize(const float* v, size_t n, float peak, float* out);
void or_cells(const float* xy, size_t n, uint32_t w, uint32_t h, uint32_t radius, uint32_t* cell_ids);
/* One neighbour-mean pass over caller positions; movable[i] != 0 marks
 * non-endpoint samples. */
void or_neighbor_mean(const float* xy, const uint8_t* movable, size_t n, uint32_t w, uint32_t h,
                      uint32_t radius, int mode, int threads, float* out_xy, uint32_t* neighbors);
/* Bounded CPU-baseline sample: the mean of the first ceil(n / stride) samples
 * only (others copied), same arithmetic as or_neighbor_mean mode 0. Returns the
 * number of samples whose mean was computed; seconds[0] receives the time of
 * the whole-set grid index, seconds[1] the time of the call (index + means). */
size_t or_neighbor_mean_sample(const float* xy, const uint8_t* movable, size_t n, uint32_t w, uint32_t h,
                               uint32_t radius, size_t stride, int threads, float* out_xy, double* seconds);

/* Distortion (src/distortion.rs). Curves are f32 pairs. */
int or_squared_integral(const float* original, size_t n_original, const float* current,
                        size_t n_current, double* out);
/* Equal-edge aggregate over edges (paths as in or_get_paths) of two snapshots. */
int or_distortion(const uint32_t* paths, uint32_t n_paths, const float* original_xy,
                  const float* current_xy, uint32_t size, double* distortion, double* rms_pixels);

/* One density-gradient advection step (an extension beyond the reference):
 * every sample that is not the first or last of its path (edge_ids differ at
 * path boundaries) moves `step` texels up the gradient of `density` (w*h,
 * the normalised map), then relaxes towards the mean of its advected path
 * neighbours by `smooth`. */
void or_advect(const float* xy, const uint32_t* edge_ids, size_t n, const float* density, uint32_t w, uint32_t h,
               float step, float smooth, float* out_xy);

/* Path rasterisation and the noisiness count (render.cpp): RGBA8 of w*h
 * pixels and the number of pixels whose RGB differs from the background.
 * palette 0 viridis, 1 cividis, 2 plasma, 3 batlow; msaa 1, 2 or 4; paths
 * (3 u32 per edge: point offset, segment offset, count) give the endpoint
 * dots when endpoint_dots is set. Returns 0 on success. */
float or_half_round(float v);   /* f32 -> f16 (nearest even) -> f32 */
int or_render(const float* xy, const uint32_t* edge_ids, const uint32_t* segments, uint32_t n_segments,
              uint32_t n_edges, const float* density, uint32_t w, uint32_t h, int color_by_edge, int palette,
              int msaa, const uint32_t* paths, uint32_t n_paths, int endpoint_dots, uint8_t* rgba,
              uint64_t* colored);

#ifdef __cplusplus
}
#endif
