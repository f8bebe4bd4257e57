/*
 * cutcell_b200.h -- C ABI of libcutcell_b200.so, the sm_100a backend for the
 * `update_cache!` hot path of CutCellMethods.jl (v0.3.0).
 *
 * Every entry point takes plain pointers and sizes. Cell columns, nodal phi,
 * PLIC plane arrays and tree leaf arrays are DEVICE pointers owned by the
 * caller (a Julia CuArray, a torch tensor): the library never frees them.
 * The library owns only its own scratch (the marching-cubes tiling table,
 * reduction partials, work lists), behind an opaque `cc_handle` that the
 * caller creates at allocate_cache time and destroys in a finalizer.
 *
 * Memory layout written (the reference's StructArray of CutCellData, one
 * plain array per field, column-major over grid.n with x fastest):
 *   kind                int8  [ncell]
 *   ambiguous           uint8 [ncell]          (Julia Bool)
 *   volume_fraction     T     [ncell]
 *   centroid            T     [D*ncell]        (D contiguous per cell)
 *   face_fraction       T     [2D*ncell]       (-x,+x,-y,+y,-z,+z per cell)
 *   face_centroid_local T     [2D*(D-1)*ncell] (per direction, in-plane axes
 *                                               in increasing order)
 *   interface_centroid  T     [D*ncell]
 *   phi                 T     [prod(n+1)]      (nodal block, x fastest)
 * (reference: src/cut_cell.jl:112-120, src/cache.jl:101-105,
 *  src/marching_squares/cache.jl:41-47, src/marching_cubes/cache.jl:30-36)
 *
 * All update entry points are asynchronous on `stream` (a cudaStream_t, or
 * NULL for the legacy default stream); the Julia/Python shims synchronize
 * before returning, as the reference's update_cache! does
 * (src/marching_squares/cache.jl:62).
 */
#ifndef CUTCELL_B200_H
#define CUTCELL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------
 * Mirrors the reference's host-side validation:
 *   CC_DIM_MISMATCH      DimensionMismatch, src/cache.jl:107-121,
 *                        src/marching_squares/cache.jl:140-147
 *   CC_ANISOTROPIC       ArgumentError, src/plic/surface.jl:41-45
 *   CC_BACKEND_MISMATCH  ArgumentError, src/marching_squares/cache.jl:119-121
 */
typedef enum {
  CC_OK = 0,
  CC_DIM_MISMATCH = 1,
  CC_ANISOTROPIC = 2,
  CC_BACKEND_MISMATCH = 3,
  CC_BAD_TAPE = 4,
  CC_DEVICE_TIMEOUT = 5,
  CC_CUDA_ERR = 6,
  CC_BAD_ARG = 7,
  CC_BAD_TABLE = 8,
  CC_NO_TABLE = 9,
  CC_TOO_LARGE = 10,
  CC_BAD_FILE = 11
} cc_status;

/* Precision of a cache: the element type T of its columns. CC_MIXED stores Float32 columns and
 * evaluates in Float32 with Float64 islands: the edge root phi_a / (phi_a - phi_b) when the
 * Float32 denominator is below 2^-100; the marching-cubes asymptotic face and interior deciders
 * (exact signs: products of Float32 values are exact in Float64); PLIC's plane-cube clips
 * (gvf2 / gvf3). calc_volume and the report reduce in compensated Float64 in every precision.
 * The learned correction does not take CC_MIXED handles. */
typedef enum { CC_F32 = 0, CC_F64 = 1, CC_MIXED = 2 } cc_prec;

/* Methods (the reference's stateless method tags). */
typedef enum {
  CC_MARCHING_SQUARES = 0, /* src/marching_squares/marching_squares.jl:68 */
  CC_MARCHING_CUBES = 1,   /* src/marching_cubes/marching_cubes.jl:53    */
  CC_PLIC = 2              /* src/plic/plic.jl:30                         */
} cc_method;

/* A CartesianGrid{D}: origin x0, cell size d, cells per axis n. Node i (0-based)
 * along axis a sits at  T(x0[a]) + T(i) * T(d[a])  with no FMA contraction
 * (the get_node expression; the grid is narrowed to T once, as
 * `convert(CartesianGrid{D,T}, grid)` at src/marching_squares/cache.jl:58). */
typedef struct {
  int32_t dim; /* 2 or 3 */
  int32_t pad_;
  double x0[3];
  double d[3];
  int64_t n[3]; /* cells per axis; n[2] = 1 in 2D */
} cc_grid;

/* Column pointers of a cache (device). Unused in a call may be NULL only
 * where the entry point says so. */
typedef struct {
  int8_t* kind;
  uint8_t* ambiguous;
  void* volume_fraction;
  void* centroid;
  void* face_fraction;
  void* face_centroid_local;
  void* interface_centroid;
} cc_cells;

/* ---- the body: a CSG tree flattened to a postfix op-tape -----------------
 * Each op evaluates a primitive at the sample point (or, for CC_OP_NONE,
 * pops the stack) and combines the value into the stack:
 *   PUSH  push v                MIN   top = (v < top) ? v : top
 *   MAX   top = (v > top)? v:top   SMIN top = polynomial smooth-min(top, v, k)
 *   SUB   top = max(top, -v)    NEG   top = -top (CC_OP_NONE only, no pop)
 * Parameters are doubles in `params`, narrowed to the cache's T at launch.
 * Stands in for SDFLibrary.jl's sdf_value/get_sdf (called at
 * src/marching_squares/cache.jl:69, src/plic/plic.jl:74). */
enum {
  CC_OP_NONE = 0,   /* no primitive: pop v, then combine                    */
  CC_OP_SPHERE = 1, /* D=3: cx cy cz r  | D=2 (circle): cx cy r           */
  CC_OP_BOX = 2,    /* c[D] h[D] (half extents, axis aligned)              */
  CC_OP_TORUS = 3,  /* D=3: c[3] R[9] (row major, local = R*(x-c)) Rmaj rmin */
  CC_OP_PLANE = 4,  /* p[D] n[D]: dot(n, x - p)                            */
  CC_OP_TRIG = 5,   /* a k[D] c: a * prod_i sin(k_i x_i) + c               */
  CC_OP_CONST = 6,  /* v (SDFLibrary's EmptyGeo(v))                        */
  CC_OP_STAR = 7,   /* D=2: cx cy r0 a[5] ph[5]: |x-c| - (r0 + sum_k a_k cos(k th + ph_k)), k=2..6 */
  CC_OP_COUNT = 8
};
enum {
  CC_COMB_PUSH = 0,
  CC_COMB_MIN = 1,
  CC_COMB_MAX = 2,
  CC_COMB_SMIN = 3,
  CC_COMB_SUB = 4,
  CC_COMB_NEG = 5
};
#define CC_TAPE_MAX_OPS 256
#define CC_TAPE_MAX_PARAMS 1024
#define CC_TAPE_MAX_STACK 8

typedef struct {
  uint8_t opcode;  /* CC_OP_* */
  uint8_t combine; /* CC_COMB_* */
  uint16_t poff;   /* first parameter of the primitive */
  uint16_t kparam; /* parameter index of k for CC_COMB_SMIN */
  uint16_t reserved;
} cc_op;

typedef struct {
  const cc_op* ops; /* host pointer */
  int32_t n_ops;
  int32_t n_params;
  const double* params; /* host pointer */
} cc_optape;

/* ---- marching-cubes tiling table ------------------------------------------
 * A flat, position-independent blob that encodes the per-cube Lewiner
 * dispatch of src/marching_cubes/marching_cubes.jl:538-651: per lookup index
 * (bit p set when corner p+1 is outside, src/marching_cubes/marching_cubes.jl:343-349)
 * the case number, up to six signed face tests (the asymptotic decider,
 * :401-406), one outcome per combination of test results, each naming an
 * optional interior test (:427-504) and the tiling(s) it selects. The Julia
 * shim encodes MarchingCubes.jl's own tables into it; the package can also
 * generate a project-designed tiling in the same format.
 *
 *   header  : cc_mc_table_header
 *   luts    : cc_mc_lut[256]
 *   outcomes: cc_mc_outcome[n_outcomes]
 *   tiles   : cc_mc_tile[n_tiles]
 *   codes   : uint8_t[n_codes]   (edge codes 1..13, three per triangle)
 */
#define CC_MC_TABLE_MAGIC 0x544D4343u /* 'CCMT' */
typedef struct {
  uint32_t magic;
  uint32_t version; /* 1 */
  uint32_t n_outcomes;
  uint32_t n_tiles;
  uint32_t n_codes;
  uint32_t total_bytes;
} cc_mc_table_header;
typedef struct {
  uint8_t lcase;  /* MarchingCubes.cases[lut][1]: 1..15 */
  uint8_t ntests; /* 0..6 face tests */
  int8_t face[6]; /* signed face codes, MarchingCubes.jl face numbering */
  uint16_t outcome_base;
  uint16_t pad_;
} cc_mc_lut;
enum { CC_MC_INTERIOR_NONE = 0, CC_MC_INTERIOR_CASE4_10 = 1, CC_MC_INTERIOR_EDGE = 2 };
typedef struct {
  uint8_t itype; /* CC_MC_INTERIOR_* */
  uint8_t edge;  /* 0-based reference edge for CC_MC_INTERIOR_EDGE */
  int8_t s;      /* sign handed to the interior test */
  uint8_t pad_;
  uint16_t tile_true;  /* tiling when there is no interior test, or it holds */
  uint16_t tile_false; /* tiling when the interior test fails */
} cc_mc_outcome;
typedef struct {
  uint16_t code_off;
  uint8_t ntris;
  uint8_t pad_;
} cc_mc_tile;

/* ---- handle -------------------------------------------------------------- */
typedef struct cc_handle cc_handle;

/* Create the library-side state for one cache (the reference's
 * allocate_cache, src/cache.jl:29). `n` is cells per axis. Allocates the
 * handle's device scratch on `device`. */
cc_status cc_handle_create(int32_t device, int32_t method, int32_t dim, int32_t prec,
                           const int64_t n[3], cc_handle** out);
cc_status cc_handle_destroy(cc_handle* h);
/* The number of mbarrier polls after which a wait of the learned kernels (for a CTA's own
 * tensor-core MMAs) gives up, for later launches; returns the previous value. A negative value
 * restores the default (2^22). Lowering it to 0 makes every such wait give up at once: a way to
 * exercise the timeout path, which then reports CC_DEVICE_TIMEOUT. */
int64_t cc_set_wait_limit(int64_t polls);
/* Upload a marching-cubes tiling table blob (validated) into the handle. */
cc_status cc_handle_set_mc_table(cc_handle* h, const void* blob, size_t nbytes);

/* Marching cubes, fused: sample phi at every node from the op-tape and build
 * every cell's CutCellData{3,T,6,2} (src/marching_cubes/cache.jl:38-39 ->
 * src/marching_squares/cache.jl:55-78). phi is T[prod(n+1)]. */
cc_status cc_mc_update(cc_handle* h, const cc_grid* g, const cc_optape* body, void* phi,
                       const cc_cells* cells, void* stream);
/* Marching cubes from a caller-supplied nodal field (the cell pass alone,
 * src/marching_squares/cache.jl:75-78): phi is read, not written. */
cc_status cc_mc_cells_from_phi(cc_handle* h, const cc_grid* g, const void* phi,
                               const cc_cells* cells, void* stream);

/* Marching squares on a CartesianGrid{2} (src/marching_squares/cache.jl:49-78). */
cc_status cc_ms_update(cc_handle* h, const cc_grid* g, const cc_optape* body, void* phi,
                       const cc_cells* cells, void* stream);
cc_status cc_ms_cells_from_phi(cc_handle* h, const cc_grid* g, const void* phi,
                               const cc_cells* cells, void* stream);

/* Marching squares on the leaves of an AdaptiveMesh{2}
 * (src/marching_squares/cache.jl:115-137). Leaf i has `level[i]` and integer
 * coordinates (coord[2i], coord[2i+1]) at that level; its size is
 * base_d / 2^level and its corners x0 + T(coord + bit) * h
 * (src/marching_squares/marching_squares.jl:113-121). level/coord are device
 * int32 arrays; phi4 is T[4*nleaves] (MS_NODE_BITS order per leaf). */
typedef struct {
  double x0[2];
  double base_d[2];
  int64_t nleaves;
  const int32_t* level;
  const int32_t* coord;
} cc_tree;
cc_status cc_ms_tree_update(cc_handle* h, const cc_tree* t, const cc_optape* body, void* phi4,
                            const cc_cells* cells, void* stream);

/* PLIC (src/plic/cache.jl:77-162): the fit pass writes normals (D*T per cell),
 * intercepts, is_valid, volume_fraction and kind; the face pass writes the
 * resolved face_fraction. centroid / face_centroid_local / interface_centroid
 * / ambiguous are not touched (NaN / false from allocation). */
cc_status cc_plic_update(cc_handle* h, const cc_grid* g, const cc_optape* body,
                         const cc_cells* cells, void* normals, void* intercepts,
                         uint8_t* is_valid, void* stream);

/* calc_volume (src/volume.jl:29-40): sum over cells of the PLIC solid
 * fraction times prod(d), accumulated on the device in compensated Float64.
 * Blocking; writes the result to *out. */
cc_status cc_calc_volume(cc_handle* h, const cc_grid* g, const cc_optape* body, double* out,
                         void* stream);

/* Monte Carlo measure of {phi < 0} inside the box lo..hi (3D): n_points seeded points, point p's
 * coordinates three successive splitmix64 outputs of (seed XOR (3p + axis)) as 53-bit fractions of
 * the box; the body is evaluated in Float64. An independent check of calc_volume; no counterpart
 * in the reference. Blocking; *inside counts the points inside, *volume (if not NULL) is
 * inside / n_points times the box volume. */
cc_status cc_monte_carlo_volume(cc_handle* h, const cc_optape* body, const double lo[3], const double hi[3],
                                int64_t n_points, uint64_t seed, int64_t* inside, double* volume, void* stream);

/* cut_cell_report (src/cut_cell.jl:302-319) over a cache's columns.
 * Blocking. counts = {n, cut, inside, outside, ambiguous}. */
cc_status cc_report(cc_handle* h, int64_t ncell, const int8_t* kind, const uint8_t* ambiguous,
                    const void* volume_fraction, int64_t counts[5],
                    double* min_volume_fraction, void* stream);

/* generate_mesh for a marching-cubes cache (src/marching_cubes/surface.jl:82-112), on the device:
 * the surface its cut cells integrate -- each cut cell's triangles the tile its moments used, a
 * vertex on a grid edge that edge's crossing as the cells place it (anchored on the outside node),
 * shared by every cell around the edge, code 13 the cell's interior vertex (the mean of its
 * crossings). Watertight inside the grid, open at its bounds, wound so each triangle's normal
 * points out of the body. `phi` is the cache's nodal field. vertices T[n_vertices][3],
 * triangles int32[n_triangles][3] (0-based vertex indices), triangle_cells int64[n_triangles]
 * (the cell of each triangle; may be NULL). Order: edge vertices by lower node (linear, x fastest)
 * then axis x, y, z; then interior vertices by cell; triangles by cell, each cell's in tile order.
 * Call with vertices = triangles = NULL to count; then with arrays of at least the counted
 * sizes. Blocking. The handle keeps the counting call's per-block results: an emitting call that
 * follows it with the same phi pointer and grid, and no update in between, skips the second
 * count. phi must not be written between the two calls; an emit that would then run past the
 * counted capacities writes nothing beyond them and returns CC_BAD_ARG. Scratch kept on the
 * handle: 4 bytes per node, plus about 1 byte per node and per cell for the kept counts. */
cc_status cc_mc_mesh(cc_handle* h, const cc_grid* g, const void* phi, void* vertices, int64_t vertex_capacity,
                     int32_t* triangles, int64_t triangle_capacity, int64_t* triangle_cells,
                     int64_t* n_vertices, int64_t* n_triangles, void* stream);
/* cell_indices (src/marching_cubes/surface.jl:128-143): each triangle's cell, 0-based linear index,
 * from its centroid floored against the grid (in Float64), clamped to the grid. Blocking. */
cc_status cc_mc_mesh_cell_indices(cc_handle* h, const cc_grid* g, const void* vertices, const int32_t* triangles,
                                  int64_t n_triangles, int64_t* cells, void* stream);

/* generate_mesh for a marching-squares cache (src/marching_squares/surface.jl:70-111), on the device:
 * the contour of the cache's phi -- a grid's nodal block, or a tree's per-leaf corners -- as the
 * cells' cell_interface segments (oriented out of the body) in cell (leaf) order, vertices welded
 * by exact coordinate equality and numbered by first occurrence (segment order, start before end),
 * the numbering of the reference's serial weld. The contour is built into the handle (blocking);
 * *n_vertices and *n_segments receive its size. cc_ms_mesh_fetch then copies it out: vertices
 * T[n_vertices][2], segments int32[n_segments][2] (0-based), cells int64[n_segments] (each
 * segment's cell or leaf; any pointer may be NULL). No device fault on any input: every hash probe
 * is bounded. */
cc_status cc_ms_mesh_grid(cc_handle* h, const cc_grid* g, const void* phi, int64_t* n_vertices, int64_t* n_segments,
                          void* stream);
cc_status cc_ms_mesh_tree(cc_handle* h, const cc_tree* t, const void* phi4, int64_t* n_vertices, int64_t* n_segments,
                          void* stream);
cc_status cc_ms_mesh_fetch(cc_handle* h, void* vertices, int32_t* segments, int64_t* cells, void* stream);

/* extract_surface_plic (src/plic/surface.jl:48-97 in 2D, :119-185 in 3D), on the device: the
 * planes n . xi = a of n_entries cells (in each cell's unit frame, as a PLIC cache stores them)
 * clipped to their cells. 3D: the polygon of the plane's crossings with the cube's edges (a corner
 * on the plane taken once), ordered by angle about its centroid in the plane's basis
 * (surface.jl:239-267) and fanned from its first vertex; a fan triangle with
 * |cross|^2 < (2 min_tri_area_fraction min(d)^2)^2 is dropped, a polygon of fewer than 3 points
 * draws nothing. 2D: one segment per entry, dropped when shorter than
 * min_tri_area_fraction * min(d); an entry whose line does not cross its cell draws a zero-length
 * segment. Entries contribute in order, and no node is shared between entries.
 *   prec        CC_F32 / CC_MIXED (float planes and output) or CC_F64 (double).
 *   normals     T[n_entries][D], intercepts T[n_entries], is_valid uint8[n_entries] or NULL (NULL:
 *               a zero normal marks a degenerate fit, which draws nothing in 3D and a zero-length
 *               segment in 2D).
 *   cell_index  int64[n_entries], the linear (x-fastest, 0-based) cell of each entry; NULL means
 *               every cell of g in order (n_entries is then ignored).
 * Output: nodes T[n_nodes][D], elements int32[n_elements][D] (0-based: triangles in 3D, segments
 * in 2D), element_cells int64[n_elements] (the cell each element was drawn for). Call with
 * nodes = elements = NULL to count, then with arrays of at least the counted sizes. Blocking. */
cc_status cc_plic_surface(int prec, const cc_grid* g, const void* normals, const void* intercepts,
                          const uint8_t* is_valid, const int64_t* cell_index, int64_t n_entries,
                          double min_tri_area_fraction, void* nodes, int64_t node_capacity, int32_t* elements,
                          int64_t element_capacity, int64_t* element_cells, int64_t* n_nodes, int64_t* n_elements,
                          void* stream);

/* generate_mesh for a PLIC cache (src/plic/surface.jl:28-37): cc_plic_surface over every cell of the
 * cache's grid, from the cache's own normals / intercepts / is_valid (the grid is checked against
 * the cache's size). The handle keeps what the counting call found -- the entries that draw, their
 * clipped polygons and the scanned offsets: an emitting call that follows it with the same arrays,
 * grid and fraction, and no update in between, writes that counted surface without clipping
 * again. It is the surface of the planes as they were at the count, so planes written in place
 * between the two calls do not reach the output. */
cc_status cc_plic_mesh(cc_handle* h, const cc_grid* g, const void* normals, const void* intercepts,
                       const uint8_t* is_valid, double min_tri_area_fraction, void* nodes, int64_t node_capacity,
                       int32_t* elements, int64_t element_capacity, int64_t* element_cells, int64_t* n_nodes,
                       int64_t* n_elements, void* stream);

/* ---- batched marching squares -----------------------------------------------------------
 * Many MarchingSquaresCutCell updates (update_cache! on a CartesianGrid,
 * src/marching_squares/cache.jl:49-78, or on an AdaptiveMesh{2}'s leaves, :115-137), each with
 * its own body and columns, in ONE persistent launch over a work list of grid tiles and leaf
 * chunks, replayed from a CUDA graph. No counterpart entry point in the reference, which runs one
 * update per call. Each item's results are bit-identical to cc_ms_update / cc_ms_tree_update on
 * the same inputs, whatever the launch shape. The batch stores the items' device pointers; they
 * must stay valid while the batch is run. */
typedef struct cc_batch cc_batch;
typedef struct {
  int32_t tile_x, tile_y; /* grid tile in cells (1..256 each, at most 4096 cells) */
  int32_t threads;        /* per CTA: a multiple of 32 in 32..256; also the leaves per tree chunk */
  int32_t ctas_per_sm;    /* persistent CTAs per SM (148 SMs) */
  int32_t chunk;          /* tiles taken per atomic pop */
  int32_t use_graph;      /* replay a captured CUDA graph (1) or launch directly (0) */
  int32_t band_percent;   /* band compaction, 0..100: a grid tile whose cut cells are at most this
                           * percent of its cells fills its uncut cells first and then builds the
                           * cut ones densely (0 never, 100 always); results are the same bits */
} cc_batch_config;
cc_status cc_batch_create(int32_t device, int32_t prec, cc_batch** out);
cc_status cc_batch_destroy(cc_batch* b);
/* Add an update; *item (if not NULL) receives its index. The body must be a 2D op-tape. */
cc_status cc_batch_add_ms_grid(cc_batch* b, const cc_grid* g, const cc_optape* body, void* phi,
                               const cc_cells* cells, int32_t* item);
cc_status cc_batch_add_ms_tree(cc_batch* b, const cc_tree* t, const cc_optape* body, void* phi4,
                               const cc_cells* cells, int32_t* item);
/* Move an item's body: the same op structure with new parameters (CC_BAD_TAPE otherwise). Waits
 * for the batch's previous run; the next run uses the new parameters. */
cc_status cc_batch_set_body(cc_batch* b, int32_t item, const cc_optape* body);
cc_status cc_batch_set_config(cc_batch* b, const cc_batch_config* cfg);
cc_status cc_batch_get_config(const cc_batch* b, cc_batch_config* cfg);
/* Items, and the work list's tiles for the current configuration (-1 before the first run). */
cc_status cc_batch_info(const cc_batch* b, int64_t* n_items, int64_t* total_tiles);
/* Run every update, ordered after the work already on `stream` and before what follows it. */
cc_status cc_batch_run(cc_batch* b, void* stream);
/* Time every candidate launch shape (tiles 32x4..128x2, 128/256 threads, 2/4/8 CTAs per SM,
 * chunks 1/4, band compaction 0/25/100 percent) on the batch as it stands, `reps` timed runs
 * each, and keep the fastest. */
cc_status cc_batch_autotune(cc_batch* b, int32_t reps, cc_batch_config* best, float* best_ms, void* stream);

/* ---- learned volume-fraction correction ----------------------------------------------------
 * An MLP 8 -> 64 -> 64 -> 1 (GELU hidden layers, sigmoid output p; tensor-core GEMMs on BF16
 * operands with FP32 accumulate) that corrects marching cubes' fluid volume fraction of a cut
 * cell from its corner values over the cell size, x = phi / d[0] in MC_NODE_BITS order. There is
 * no counterpart function in the reference, whose plain marching cubes
 * (src/marching_cubes/moments.jl:275-346) this corrects. The correction is first order in the
 * curvature: with quad(x) the projection of x on the four non-linear corner patterns (xy, xz,
 * yz, xyz of the -1/+1 corner bits) and lin(x) = x - quad(x), the network sees
 *     x~ = lin(x) + quad(x) * CC_MLP_CURVATURE_NORM / |quad(x)|
 * and the cell's fraction becomes
 *     corrected = plain + s * CC_MLP_CORRECTION_SCALE * (2 p(x~) - 1),  s = |quad(x)| / CC_MLP_CURVATURE_NORM
 * (planar cells, quad = 0, keep the plain value). It is trained on the fluid fractions of
 * marching cubes at 8x sub-refinement. The inputs, the first-layer weights, the hidden
 * activations and the second-layer weights enter the GEMMs as BF16 high + low pairs (hi*hi +
 * lo*hi + hi*lo), about 16 significant bits.
 * Parameters: FP32, CC_MLP_NPARAM of them: W1[64][8] b1[64] W2[64][64] b2[64] w3[64] b3. */
#define CC_MLP_NPARAM 4801
#define CC_MLP_MAX_TILES 1184
#define CC_MLP_CORRECTION_SCALE 0.0625f
#define CC_MLP_CURVATURE_NORM 0.02f
typedef struct cc_mlp cc_mlp;
cc_status cc_mlp_create(int32_t device, cc_mlp** out);
cc_status cc_mlp_destroy(cc_mlp* m);
/* host <-> device parameters; setting them also resets the Adam moments and step */
cc_status cc_mlp_set_params(cc_mlp* m, const float* params, int32_t n);
cc_status cc_mlp_get_params(cc_mlp* m, float* params, int32_t n);
/* `steps` Adam steps (learning rate lr) on device samples feats[n][8]. With plain fractions
 * (plain != NULL) the loss is the mean of w[i] |c_i - (labels[i] - plain[i])|, c_i the
 * correction above; with plain NULL it is the mean of w[i] (p_i - labels[i])^2 on the raw
 * features (the network alone). w = weights, or 1 where weights is NULL. Each step draws
 * tiles*128 samples by a counter-based hash of (seed, step, slot); with augment != 0 the same
 * hash also picks one of the 48 symmetries of the cube per sample and permutes its corner values
 * accordingly. Blocking; *last_loss receives the final step's loss. */
cc_status cc_mlp_train(cc_mlp* m, const float* feats, const float* labels, const float* plain,
                       const float* weights, int64_t n, int32_t steps, int32_t tiles, float lr, uint64_t seed,
                       int32_t augment, float* last_loss, void* stream);
/* The gradient (summed over tiles) and loss of one step's sample draw, without updating: for
 * checking the backward kernels. grad is a host array of CC_MLP_NPARAM floats. */
cc_status cc_mlp_grad(cc_mlp* m, const float* feats, const float* labels, const float* plain, const float* weights,
                      int64_t n, int32_t tiles, uint64_t seed, int32_t step, int32_t augment, float* grad,
                      float* loss, void* stream);
/* For device features feats[n][8]: the network output p of the raw features (correction == 0),
 * or the correction s * CC_MLP_CORRECTION_SCALE * (2 p(x~) - 1) (correction != 0). */
cc_status cc_mlp_predict(cc_mlp* m, const float* feats, int64_t n, int32_t correction, float* out, void* stream);
/* Read a weights file into the host array params[n] (n = CC_MLP_NPARAM), checking it: a 64-byte
 * little-endian header -- magic "CCB2MLP1", u32 version 1, u32 parameter count, f32
 * CC_MLP_CORRECTION_SCALE, f32 CC_MLP_CURVATURE_NORM, u64 FNV-1a-64 of the parameter bytes, 32
 * zero bytes -- then the FP32 parameters. Host only (no device is touched); CC_BAD_FILE when the
 * file is missing, short, or any field or the checksum disagrees. */
cc_status cc_mlp_read_weights(const char* path, float* params, int32_t n);
/* Training samples from the cut cells of the last update on h (a Float32 marching-cubes handle):
 * feats[i][8] = corner phi / d[0], plain[i] = its plain volume fraction, labels[i] = the fluid
 * fraction of marching cubes at 8x sub-refinement of `body` (Float64), index[i] (if not NULL) =
 * the cell's linear index. Blocking; at most `capacity` cells, *count receives how many were
 * written. */
cc_status cc_mc_learned_samples(cc_handle* h, const cc_grid* g, const cc_optape* body, const void* phi,
                                const cc_cells* cells, float* feats, float* labels, float* plain, int64_t* index,
                                int64_t capacity, int64_t* count, void* stream);
/* cc_mc_update with the learned correction of cut cells' volume fractions. A cut cell keeps its
 * plain value where p is not finite, the correction's magnitude exceeds `bound` (a negative
 * bound rejects every prediction) or the corrected fraction leaves [0, 1]; *n_fallback (if not
 * NULL; then blocking) receives how many cut cells kept the plain value. */
cc_status cc_mc_update_learned(cc_handle* h, const cc_grid* g, const cc_optape* body, void* phi,
                               const cc_cells* cells, const cc_mlp* mlp, float bound, int64_t* n_fallback,
                               void* stream);

/* Marching cubes from a caller-supplied nodal field WITHOUT allocating: no counterpart in the
 * reference. For callers that may not let a library allocate device memory -- a solver whose
 * device memory comes from its own pool, budgeted up front, or a time-stepping loop where a
 * cudaMalloc (which can synchronize the device) mid-step is not acceptable. Same inputs and
 * outputs as cc_mc_cells_from_phi, plus the device index, the precision (CC_F32 / CC_F64) and the
 * tiling table as a HOST blob (validated, then copied into the library's static scratch). No
 * handle: the scratch (the table's device copy and the cut-band work list) is one file-scope
 * __device__ array of 32 MiB + 64.25 KiB that every GPU loading the library holds until exit.
 *   - Grids of more than 8,388,608 (2^23) cells are rejected with CC_TOO_LARGE.
 *   - Every call looks up that array's device address (cudaGetSymbolAddress) with `device`
 *     current. The first call on a device also loads the library's device code there: make
 *     that first call before any stream capture.
 *   - The table is copied from the host only when the device does not already hold the same
 *     blob (compared by size and hash) from an earlier call in the same context.
 *   - Every call reuses the same array: calls that overlap on the GPU (other streams, other host
 *     threads) race. Serialize them, e.g. on one stream.
 * Calls no cudaMalloc, cudaFree or other allocating routine. */
cc_status cc_mc_cells_from_phi_noalloc(int32_t device, int32_t prec, const cc_grid* g, const void* table,
                                       size_t table_bytes, const void* phi, const cc_cells* cells,
                                       void* stream);

/* Library version string. */
const char* cc_version(void);
/* Last CUDA error text seen by the library on this thread ("" if none). */
const char* cc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* CUTCELL_B200_H */
