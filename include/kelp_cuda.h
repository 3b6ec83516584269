/*
 * kelp_cuda.h -- C ABI of the B200 (sm_100a) implementation of KELP's
 * compiled time-stepping path.
 *
 * The library owns all device memory.  A context binds one CUDA device and
 * one stream; it holds the resident mesh (node table, element table,
 * node->element CSR, grid hash), a small ring of velocity snapshots, and the
 * particle state.  Calls on one context are not thread-safe; callers
 * serialise them.  Every function returns 0 on success or a KC_ERR_* code;
 * kc_last_error() gives the message.  Invalid arguments are rejected on the
 * host before any kernel runs.  Per-particle failures are data
 * (status OUTSIDE + failure reason), as in the reference.
 *
 * Reference interfaces replaced (paths inside the KELP project):
 *   kc_step / kc_run   <- integrators.rk2_step / rk4_step / euler_step
 *                         (src/kelp/numerics/integrators.py:5611, :6013, :5150),
 *                         the per-step call of tracking.run_single_realization
 *                         (src/kelp/tracking.py:2643-2655)
 *   kc_mesh_upload     <- the arrays of core.mesh.Mesh after build_search
 *                         (src/kelp/core/mesh.py:40-166, :844-1001)
 *   kc_field_upload    <- core.io.VelocityField snapshot arrays
 *                         (src/kelp/core/io.py:180)
 *   kc_particles_*     <- core.particles.ParticleState arrays
 *                         (src/kelp/core/particles.py:153)
 *   kc_node_xyz_fill   <- core.mesh._node_xyz_fill (src/kelp/core/mesh.py:712)
 *   kc_find_nearest    <- core.mesh.find_nearest_nodes (src/kelp/core/mesh.py:1896)
 *   kc_find_elements   <- core.mesh.find_containing_elements (src/kelp/core/mesh.py:2286)
 *   kc_find_elements_walk <- core.mesh.find_containing_elements_walk
 *                         (src/kelp/core/mesh.py:2631-2712)
 *   kc_elem_neighbors_upload <- core.mesh.build_elem_neighbors (src/kelp/core/mesh.py:2824)
 *   kc_field_upload_async <- the snapshot upload of tracking.run_single_realization, overlapped
 *                         with the steps (tracking.py:2947, the next bracket's records)
 *   kc_elem_centers_upload <- the mesh's elem_center_lon / elem_center_lat, read by
 *                         numerics.interpolate._interp_leastsq_core (interpolate.py:52)
 *   kc_sigma_upload    <- core.mesh.Mesh.sigma with vertical_coord "sigma" (src/kelp/core/mesh.py:63-91)
 *   kc_cgrid_upload    <- the C-grid tables of readers.nemo._mesh.build_nemo_cgrid_mesh
 *                         (src/kelp/readers/nemo/_mesh.py:16-264), read by
 *                         numerics.nemo_cgrid (src/kelp/numerics/nemo_cgrid.py:84-512)
 *   kc_field_upload_eta <- core.io.VelocityField.eta (src/kelp/core/io.py:180)
 *   kc_rng_normals     <- numerics.diffusion._normal_pair (src/kelp/numerics/diffusion.py:233)
 *   kc_sample_field    <- numerics.sampling.sample_field (src/kelp/numerics/sampling.py:727)
 *   kc_sample_field_sigma <- its sigma-mesh branch _sample_sigma_3d (sampling.py:620-723)
 *   kc_beach_surface   <- the vel.eta / vel.scalars[dry_mask_var] reads of tracking._apply_beaching_hook
 *   kc_sigma_surfaces  <- the sigma_eta_start / sigma_eta_end arguments of the step functions
 *                         (src/kelp/numerics/integrators.py:1358-1441; tracking.py:2562-2596)
 *   kc_sigma_surface_slots <- tracking._eta_at_time (src/kelp/tracking.py:3097-3133) on resident records
 *   kc_grid_cell_stats <- core.mesh._gh_sample_stats, the per-sample kernel of the occupancy cell rule
 *                         choose_grid_hash_cell (src/kelp/core/mesh.py:384-461, :464-616)
 *                         (src/kelp/tracking.py:236-327)
 */
#ifndef KELP_CUDA_H
#define KELP_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define KC_ABI_VERSION 14

#define KC_OK 0
#define KC_ERR_ARG 1      /* invalid argument or combination */
#define KC_ERR_CUDA 2     /* CUDA runtime error */
#define KC_ERR_STATE 3    /* call out of order (no mesh / field / particles) */
#define KC_ERR_DEVICE 4   /* a device-side iteration cap was hit */

/* field element types */
#define KC_F32 0
#define KC_F64 1
#define KC_F16 2     /* float32 input stored as float16 with a power-of-two scale per row */

/* numerical forms of kc_step */
#define KC_PLAIN 0   /* float64 interpolation: the reference's arithmetic */
#define KC_MIXED 1   /* float32 interpolation, float64 positions and element decisions */

/* integration schemes */
#define KC_EULER 0
#define KC_RK2 1
#define KC_RK4 2

typedef struct kc_ctx kc_ctx;

typedef struct kc_mesh_desc {
    long long n_nodes;
    long long n_elems;
    int max_v;                   /* 3 or 4 columns in elem_nodes */
    int max_conn;                /* columns in node_to_elems */
    const double* nodes_lon;     /* (N) degrees */
    const double* nodes_lat;     /* (N) degrees */
    const double* depth;         /* (N) metres positive down; may be NULL for 2-D */
    const int* elem_nodes;       /* (E, max_v), -1 padded */
    const int* node_to_elems;    /* (N, max_conn), -1 padded */
    const int* node_to_elems_count; /* (N) */
    const int* gh_offsets;       /* (gh_nx * gh_ny + 1) CSR offsets */
    const int* gh_node_ids;      /* (N) node ids in hash order */
    const double* node_xyz;      /* (N, 3) unit-sphere table */
    double gh_cell_size, gh_lon_min, gh_lat_min;
    int gh_nx, gh_ny, gh_wrap_lon, gh_far_rows;
    int exact_nearest;           /* mesh.metadata["exact_nearest"] */
    double r_earth;              /* mesh.r_earth */
    const double* z_levels;      /* (n_levels) interfaces positive down, NULL for 2-D */
    int n_levels;
} kc_mesh_desc;

typedef struct kc_step_args {
    int scheme;                  /* KC_EULER / KC_RK2 / KC_RK4 */
    int dims;                    /* 2 or 3 */
    int slot_a, slot_b, slot_t;  /* bracket pair and stage target snapshots */
    double alpha0;               /* bracket fraction at the step's start */
    double alpha_k[4];           /* stage alphas c_k * dt / dt_to_next */
    double dt;                   /* seconds, > 0 */
    double time_dir;             /* +1 forward, -1 backward */
    int w_code;                  /* 3-D W: 0 nearest, 1 barycentric, 2 least squares, 3 inverse distance
                                    (2 and 3: plain form; vertical.py:493-601, :1148-1229, and on sigma
                                    meshes vertical_sigma.py:493-563, :656-905) */
    int uv_vertical;             /* 3-D u/v: 0 layer (K-1 rows), 1 depth-linear (the table's M rows) */
    int kick;                    /* split uniform-Kh random walk on/off */
    double kh_x, kh_y;           /* m^2/s */
    unsigned long long seed, real_id, step_i, pid_offset;
    long long global_step;       /* delayed-release activation step, -1 for none */
    int precision;               /* KC_PLAIN (snapshots F32/F64) or KC_MIXED (snapshots F32/F16) */
    int az_kick;                 /* vertical Az kick after the step (3-D; diffusion.az_enabled) */
    int az_field;                /* Az from the bracket slots' az rows (kc_field_upload_az), else az_const */
    double az_const;             /* m^2/s, >= 0 */
    double Dmin;                 /* sigma meshes: column floor (m, > 0; the reference's default 0.5) */
    double z0b_min;              /* sigma meshes: clearance above the bed (m, >= 0; default 0.1) */
    double alpha_end;            /* sigma meshes: blend fraction of the end-of-step surface,
                                    dt / dt_to_next (0 without a next snapshot) */
    int pchip;                   /* 1: monotone-cubic (PCHIP) stages from the 4-record stencil
                                    slot_a, slot_b, slot_t, slot_d at times pchip_t
                                    (temporal_reconstruct.py:183-325); alpha_k are then the stage
                                    times and alpha_end the end time; plain form, no Az */
    int slot_d;
    double pchip_t[4];
    int uv_lsq;                  /* element-centre u/v: 1 the least-squares plane of the anchor's elements
                                    (uv_interp "leastsq", src/kelp/numerics/interpolate.py:52-354, 644-750);
                                    2 / 3 the edge-neighbour plane with freeslip / noslip ghost values
                                    (uv_interp "edge_leastsq", interpolate.py:2588-2747; needs
                                    kc_elem_neighbors_upload).  Snapshots hold one row of E element values
                                    (3-D: u/v (K-1, E) and w (K, N) rows of stride max(E, N)); needs
                                    kc_elem_centers_upload; plain form */
} kc_step_args;

/* Beaching / resuspension of one step (src/kelp/tracking.py:199-364,
 * src/kelp/numerics/beaching.py:95-181).  Criteria flags mirror
 * beaching.criteria; resuspension: 0 never, 1 auto, 2 stochastic,
 * 3 auto_or_stochastic.  p_beach = 1 - exp(-|dt| / t_beach) and
 * p_resusp = 1 - exp(-|dt| / t_resuspend) are evaluated by the caller. */
typedef struct kc_beach_args {
    int use_depth, use_coastal, use_stochastic, on_failure;
    int resuspension, min_wet_steps;
    double depth_min, zone_depth, rewet_hysteresis, p_beach, p_resusp;
    unsigned long long seed, real_id, step_i, pid_offset;
} kc_beach_args;

int kc_abi_version(void);

/* Host routine: unit-sphere node table with the C library's cos/sin. */
int kc_node_xyz_fill(const double* lon, const double* lat, long long n, double* xyz_out);

int kc_create(int device, kc_ctx** out);
void kc_destroy(kc_ctx* ctx);
int kc_last_error(const kc_ctx* ctx, char* buf, int buflen);
int kc_synchronize(kc_ctx* ctx);

int kc_mesh_upload(kc_ctx* ctx, const kc_mesh_desc* desc);

/* The depth-linear data-point table of the mesh (uv_vertical "level" /
 * "layer_linear"): M point depths p, and per node the last usable point and
 * the bed depth (src/kelp/numerics/vertical_uv.py:181-278, :328). */
int kc_depth_points_upload(kc_ctx* ctx, int M, const double* p, const int* last, const double* bed);

/* One snapshot into ring slot `slot` (0..7): u, v (n_uv_rows, n_nodes) and
 * optional w (n_w_rows, n_nodes), all of element type `dtype` (KC_F32 or
 * KC_F64); KC_F16 takes float32 arrays and stores them as float16, each row
 * scaled by a power of two so that its largest magnitude is below 2^15. */
int kc_field_upload(kc_ctx* ctx, int slot, int dtype, long long n_nodes, int n_uv_rows,
                    const void* u, const void* v, int n_w_rows, const void* w);

/* kc_field_upload without waiting: the copies run on the library's copy
 * stream, after the last launch that read the slot, while steps already
 * launched keep running; a later step that reads the slot waits for them on
 * the device.  float32 / float64 u, v, w only (no eta or Az rows).  The host
 * arrays must stay unchanged until the copy is done (the next kc_synchronize,
 * or a step that reads the slot has finished); page-locked arrays
 * (kc_host_alloc) make the copy fully asynchronous, pageable ones are staged
 * before the call returns.  The prefetch of the tracking loop's next record
 * (tracking.py:2947 _resolve_time_bracket decides which). */
int kc_field_upload_async(kc_ctx* ctx, int slot, int dtype, long long n_nodes, int n_uv_rows, const void* u,
                          const void* v, int n_w_rows, const void* w);

/* The vertical diffusivity of the snapshot in ring slot `slot`: n_rows (= the
 * mesh's interfaces K) x n_nodes values of the slot's element type (float32
 * or float64; io.py VelocityField.az).  Uploading a new snapshot into the
 * slot drops it. */
int kc_field_upload_az(kc_ctx* ctx, int slot, int dtype, long long n_nodes, int n_rows, const void* az);

/* Particle state.  Optional pointers may be NULL (z: zeros, fr: zeros,
 * pid: the index, release_step: all released). */
int kc_particles_upload(kc_ctx* ctx, long long P, const double* lon, const double* lat,
                        const double* z, const int* status, const int* nearest_node,
                        const signed char* failure_reason, const long long* pid,
                        const int* release_step);
int kc_particles_download(kc_ctx* ctx, long long P, double* lon, double* lat, double* z,
                          int* status, int* nearest_node, signed char* failure_reason,
                          double* u, double* v, double* w);

/* Per-particle realization ids of the resident particles (NULL: every
 * particle takes kc_step_args.real_id again).  With them, the members of a
 * diffusion ensemble (tracking.py runs one realization per call of
 * run_single_realization, keyed by realization_id) share one particle array
 * and one launch: each particle's kick and beaching draws use its own id.
 * kc_particles_upload clears them; call before kc_sort. */
int kc_particles_set_realization(kc_ctx* ctx, const int* real_id);

/* A sigma mesh (FESOM-C; mesh.vertical_coord "sigma"): its K interfaces,
 * 1 at the surface to 0 at the bed, on a mesh uploaded with depth and
 * without z-levels.  3-D steps then integrate s = z / H_p in the particle's
 * column H_p = max(depth + eta, Dmin) (integrators.py:1322-1440, the sigma
 * branches of :4997-6011), in the plain form, and need every snapshot's
 * surface (kc_field_upload_eta). */
int kc_sigma_upload(kc_ctx* ctx, int K, const double* sigma);

/* The free surface eta (n_nodes float64) of the snapshot in ring slot
 * `slot`; uploading a new snapshot into the slot drops it. */
int kc_field_upload_eta(kc_ctx* ctx, int slot, long long n_nodes, const double* eta);

/* The NEMO C-grid tables of a mesh built by build_nemo_cgrid_mesh (nodes =
 * F-points, elements = T-cells with a ring of dry cells), uploaded after
 * kc_mesh_upload.  Steps on such a mesh read face-raster snapshots
 * (kc_field_upload with n_nodes = ny * nx: u, v one row in 2-D, K rows in
 * 3-D, w K + 1 rows) through the exact C-grid interpolation
 * (numerics/nemo_cgrid.py:84-222): 2-D steps as the reference's unfused
 * Euler / RK2 / RK4 with uv_interp "nemo_cgrid", 3-D steps as
 * nemo_cgrid3d_step (:416-512, fractional level coordinate, no diffusion).
 * Plain form only. */
typedef struct kc_cgrid_desc {
    int ny, nx;                  /* T / F raster shape (mesh._structured_shape) */
    int K;                       /* levels (zw has K + 1 interfaces); 0 for a 2-D mesh */
    int partial_shrunk;          /* mesh._nemo_cgrid_partial: 1 "shrunk", 0 "porous" */
    const int* corners;          /* (E, 4) node ids SW, SE, NE, NW (_nemo_cgrid_corners) */
    const long long* elem_ji;    /* (E, 2) T-cell (j, i), j, i >= 1 (_nemo_cgrid_elem_ji) */
    const int* nlev;             /* (E) wet levels, 0 for the dry ring (_nemo_cgrid_nlev) */
    const int* nlev_raster;      /* (ny * nx) wet levels per column */
    const double* e2u;           /* (ny * nx) model u-face widths, or NULL (plane edge lengths) */
    const double* e1v;           /* (ny * nx) model v-face widths, or NULL */
    const double* area;          /* 3-D: (ny * nx) T-cell areas */
    const double* zw;            /* 3-D: (K + 1) interfaces, positive down */
    const double* e3b;           /* 3-D: (ny * nx) bottom wet cell thickness */
    const int* kbu;              /* 3-D: (ny * nx) partial level of each u face, -1 none */
    const double* e3u;           /* 3-D: (ny * nx) its thickness */
    const int* kbv;              /* 3-D: (ny * nx) partial level of each v face, -1 none */
    const double* e3v;           /* 3-D: (ny * nx) its thickness */
} kc_cgrid_desc;

int kc_cgrid_upload(kc_ctx* ctx, const kc_cgrid_desc* desc);

/* Edge-neighbour table of the mesh (E x max_v int32, -1 on boundary edges;
 * entry k is the element across the edge from compacted-ring vertex k to the
 * next; src/kelp/core/mesh.py:2824-2908 build_elem_neighbors).  Needed by the
 * edge walk (elem_search: walk). */
int kc_elem_neighbors_upload(kc_ctx* ctx, int max_v, const int* elem_neighbors);

/* Element centres of the mesh (E lon, E lat in degrees: mesh.elem_center_lon /
 * elem_center_lat, src/kelp/core/mesh.py), read by the element-centre
 * least-squares u/v of kc_step_args.uv_lsq (interpolate.py:52-354). */
int kc_elem_centers_upload(kc_ctx* ctx, const double* lon, const double* lat);

/* Carried containing elements of the resident particles (P int32, -1 = no
 * guess) for elem_search "walk" (integrators.py:5019-5147, :5415-5608,
 * :5792-6011): each step walks every stage's containing element from the
 * previous stage's, hands it to the interpolation, and ends with the walked
 * element of the new position (the start element after a failed step).
 * NULL returns to the local search.  kc_particles_upload clears them; call
 * before kc_sort.  kc_particles_get_elem reads them back in upload order. */
int kc_particles_set_elem(kc_ctx* ctx, const int* elem);
int kc_particles_get_elem(kc_ctx* ctx, long long P, int* elem);

/* Containing element of each point by the local 1-ring / 2-ring scan around
 * the anchor nn[i] (NULL: the exact nearest node of the point); -1 outside. */
int kc_find_elements(kc_ctx* ctx, long long P, const double* lon, const double* lat, const int* nn, int* out);

/* Containing element of each point, walked from start[i] (-1: no guess),
 * with the widened-anchor and exact-anchor fallbacks; -1 outside. */
int kc_find_elements_walk(kc_ctx* ctx, long long P, const double* lon, const double* lat, const int* start,
                          int* out);

/* Coastal element flags (E bytes, 1 = owns a boundary edge;
 * src/kelp/core/mesh.py:2764-2821 build_boundary_info). */
int kc_coastal_upload(kc_ctx* ctx, const unsigned char* elem_is_coastal);

/* Beaching state of the resident particles: the status each had when its
 * last step began (NULL: the status the next kc_step records) and the
 * consecutive-wet-step counters (NULL: zeros).  After this call every step
 * records the entry status for the hook; kc_particles_upload clears it. */
int kc_beach_state_upload(kc_ctx* ctx, const int* prev_status, const int* wet_streak);
int kc_beach_state_download(kc_ctx* ctx, int* wet_streak);

/* The beaching hook on the resident particles after a step. */
int kc_beach(kc_ctx* ctx, const kc_beach_args* args);

/* The payload's node surfaces for the beaching hook, tracking.py:236-327 and
 * beaching.py:95-181: eta (N) the free surface added to the anchor's depth
 * (beaching.use_eta), dry_mask (N) the dry-mask variable's surface layer
 * (beaching.dry_mask_var; a node above 0.5 is dry for the depth criterion
 * and never wet for resuspension).  Each is copied and used by the following
 * kc_beach calls until set again; NULL turns it off.  The host blends them
 * as the payload does ((1 - alpha) a + alpha b).  kc_run_fused refuses a
 * beaching hook while a surface is set (it changes every step). */
int kc_beach_surface(kc_ctx* ctx, const double* eta, const double* dry_mask);

/* The tracking layer's free surfaces for the following sigma-mesh steps
 * (sigma_eta_start / sigma_eta_end of integrators.rk2_step / rk4_step /
 * euler_step, src/kelp/numerics/integrators.py:1358-1441, supplied by
 * tracking.run_single_realization, src/kelp/tracking.py:2562-2596):
 * eta_start (N) the surface at the step's start, eta_end (N) at its end, NULL
 * for the payload's own; steady 1 for a step without a next snapshot or a
 * PCHIP stencil (its stage surfaces then blend from the start towards the
 * end surface), else 0.  Copied; used by every sigma step until set again.
 * KC_ERR_STATE unless the resident mesh is a sigma mesh. */
int kc_sigma_surfaces(kc_ctx* ctx, const double* eta_start, const double* eta_end, int steady);

/* One of those surfaces (which 0: the step's start, 1: its end) evaluated on
 * the device from resident snapshot slots, as tracking._eta_at_time does
 * (src/kelp/tracking.py:3097-3133): kind 1 the eta of slots[0]; 2 the blend
 * (1 - alpha) eta(slots[0]) + alpha eta(slots[1]); 3 the monotone-cubic
 * value at time q of the four-record stencil slots[0..3] at times t[0..3]
 * (temporal_reconstruct.py:87-153); 0 turns that surface off (the payload's
 * own).  Ordered on the context's stream after pending uploads into those
 * slots.  steady as kc_sigma_surfaces. */
int kc_sigma_surface_slots(kc_ctx* ctx, int which, int kind, const int* slots, double alpha, const double* t,
                           double q, int steady);

/* Host particle arrays of kc_step_host (SoA, P entries each).  Input: lon,
 * lat, status, nearest_node required; z and failure_reason may be NULL
 * (zeros); pid (RNG particle key; NULL: the index), real_id (per-particle
 * realization; NULL: the step's) and release_step (delayed release, with
 * kc_step_args.global_step; NULL: all released) are read only from the input.
 * elem: the carried containing elements (walk mode, as kc_particles_set_elem;
 * NULL: local search), read from the input and written to the output.
 * Output: lon, lat, status, nearest_node required; z, failure_reason, u, v, w,
 * elem may be NULL (not returned).  Input and output may be the same arrays. */
typedef struct kc_host_particles {
    double* lon;
    double* lat;
    double* z;
    int* status;
    int* nearest_node;
    signed char* failure_reason;
    double* u;
    double* v;
    double* w;
    long long* pid;
    int* real_id;
    int* release_step;
    int* elem;
} kc_host_particles;

/* One step of P particles held in host memory, in the reference's per-step
 * form (state in, new state out; tracking.py:2643-2655): the particles are
 * cut into chunks of `chunk` (0: P/8, at most 64 chunks) whose upload,
 * step and download run on three streams, so the copies of one chunk overlap
 * the step of another.  Page-locked host arrays (kc_host_alloc) make the
 * copies asynchronous.  RNG keys are pid_offset + the particle's index.  The
 * particles stay resident afterwards, as after kc_particles_upload + kc_step. */
int kc_step_host(kc_ctx* ctx, const kc_step_args* args, long long P, const kc_host_particles* in,
                 const kc_host_particles* out, long long chunk);

/* One step of every resident particle; kc_run: n_steps steps in order,
 * per-step arguments, no host round trip in between. */
int kc_step(kc_ctx* ctx, const kc_step_args* args);
int kc_run(kc_ctx* ctx, const kc_step_args* steps, int n_steps);

/* One step of the resident particles [begin, begin + count) only, RNG keys
 * unchanged (a cohort of a larger array).  No reference counterpart: the
 * reference steps one cohort's state per call of its step function. */
int kc_step_range(kc_ctx* ctx, const kc_step_args* args, long long begin, long long count);

/* n_steps steps of every resident particle in ONE kernel launch: each thread
 * carries its particles through all the steps (particles are independent),
 * with the beaching hook after every step when beach != NULL (n_steps
 * argument blocks; kc_beach_state_upload first).  Same results as n_steps
 * kc_step (+ kc_beach) calls.  Every step must share dims, scheme, form and
 * snapshot element type.  With use_graph the launch is captured once as a
 * CUDA graph (argument upload + kernel) and replayed while n_steps, the
 * particle count, the mesh and the form stay the same; the per-step arguments
 * are read from a device buffer, so each replay runs the steps passed to it.
 * No reference counterpart (the reference launches one parallel loop per
 * step and per realization). */
int kc_run_fused(kc_ctx* ctx, const kc_step_args* steps, int n_steps, const kc_beach_args* beach, int use_graph);

/* Particles per block of kc_run_fused: 128 (default) or 256, both with a
 * 64-register budget (the autotuner's choice; no reference counterpart). */
int kc_set_fused_block(kc_ctx* ctx, int block);

/* Re-order the resident particles by grid-hash cell (particles that left the
 * domain last) so that a warp's particles share hash windows and elements.
 * Results do not depend on the order: every particle keeps its RNG key, and
 * kc_particles_download returns the upload order.  No reference counterpart
 * (the reference's utils/sort_seeds.py sorts seed files offline). */
int kc_sort(kc_ctx* ctx);

/* Sampling on a sigma mesh (sampling.py:620-723 _sample_sigma_3d): values
 * (rows, N) an interface field (rows == K, the sigma W interpolation of the
 * method, vertical_sigma.py:971-1031) or a mid-layer field (rows == K-1, each
 * node's column max(depth + eta, Dmin) with its mid-layer depths, z clamped to
 * it, then the method's horizontal rule); eta (N) the free surface; the other
 * arguments as kc_sample_field, methods 0 (nearest), 1 (leastsq) and 3 (idw).
 * KC_ERR_STATE unless the mesh is a sigma mesh. */
int kc_sample_field_sigma(kc_ctx* ctx, const double* values, int rows, const double* eta, double Dmin, long long P,
                          const double* lon, const double* lat, const double* z, const int* nearest,
                          const unsigned char* alive, int method, double* out);

/* Batch exact nearest node of P query points (host arrays). */
int kc_find_nearest(kc_ctx* ctx, long long P, const double* lon, const double* lat, int* out);

/* Sample a node scalar field at P points (host arrays), the rules of
 * numerics.sampling.sample_field (src/kelp/numerics/sampling.py:727-933):
 * values (N) when rows == 0, or a z-level mid-layer field (rows, N) with its
 * mid-layer depths z_mids (rows, positive down) and the points' depths z (P);
 * nearest (P) the anchors (NULL: the exact nearest node, as the reference
 * finds it), a negative anchor giving NaN; alive (P, nonzero = alive) or NULL
 * (all alive); method 0 nearest, 1 leastsq, 2 barycentric, 3 idw.  out (P)
 * receives the samples, NaN for dead or anchorless points.  The field is
 * float64, as the reference reads it; interface fields (K, N) and sigma
 * meshes are not covered (the host raises before calling).  KC_ERR_ARG for
 * a method outside 0..3, an anchor >= N or a mid-layer field without its
 * depths or the mesh depth.  z_mids NULL with rows == K: an interface field
 * (K, N) on the mesh's z-levels, sampled by the W interpolation of the
 * method as sampling.py:876-890 does (vertical.py:1330-1420). */
int kc_sample_field(kc_ctx* ctx, const double* values, int rows, const double* z_mids, long long P,
                    const double* lon, const double* lat, const double* z, const int* nearest,
                    const unsigned char* alive, int method, double* out);

/* The same batch nearest-node query, allocating nothing on the device.  For
 * callers that must not call cudaMalloc: it synchronises the whole device, and
 * it fails when the host application has already reserved the free device
 * memory for its own pool.  Queries and results are staged in one fixed
 * device array (1.25 MiB, held by every GPU that loads the library until the
 * process exits), so at most 65536 points per call (more is rejected with
 * KC_ERR_ARG).  The first call on a device looks the array's address up
 * (make it before any stream capture).  All calls share the array: calls that
 * overlap on the GPU (several contexts or threads at once) race.  Same results
 * as kc_find_nearest.  No counterpart in the reference. */
int kc_find_nearest_noalloc(kc_ctx* ctx, long long P, const double* lon, const double* lat, int* out);

/* Counter-RNG normal pairs of the diffusion kicks, drawn on the device for
 * particle ids pid_offset .. pid_offset + P - 1 and key component comp (0 the
 * horizontal pair, 1 the vertical Az kick) (out: (P, 2)).  The kick kernels
 * draw exactly these numbers, equal to the reference's bit for bit; this
 * entry point exposes them for checking
 * (src/kelp/numerics/diffusion.py:233-249 _normal_pair). */
int kc_rng_normals(kc_ctx* ctx, long long P, unsigned long long seed, unsigned long long real_id,
                   unsigned long long step_i, unsigned long long pid_offset, unsigned long long comp, double* out);

/* The grid hash of a mesh's nodes built on the device (the CSR of
 * src/kelp/core/mesh.py:844-1001 build_grid_hash): each node's cell
 * (cj * nx + ci, the quotient by cell_size truncated and clamped; lon in the
 * branch the host chose, lon_min 0 when wrap), the node ids stable-sorted by
 * cell into node_ids (n_nodes) and the CSR offsets (nx * ny + 1).  Equal to
 * the host build bit for bit. */
int kc_grid_hash_build(kc_ctx* ctx, long long n_nodes, const double* lon, const double* lat, double cell_size,
                       double lon_min, double lat_min, int nx, int ny, int wrap, int* offsets, int* node_ids);

/* One candidate cell of the grid-hash occupancy rule at P sample points
 * (host arrays; src/kelp/core/mesh.py:384-461 _gh_sample_stats, run by
 * choose_grid_hash_cell :464-616 for each cell of its ladder).  The node
 * counts of the candidate grid (cell_size, lon_min, lat_min, nx, ny, wrap:
 * the geometry the host derived for it; lon_branch (n_nodes) the node
 * longitudes in the branch the host chose, the resident mesh's latitudes)
 * and their 2-D prefix table are built on the device.  For every sample:
 * nn (P) its exact nearest node on the resident mesh's own grid hash
 * (-1 only on an empty grid; the other outputs are then 0), occ the nodes
 * in its candidate 3x3 window, approx 1 where that node lies outside the
 * window, unprov 1 where the 3x3 certificate does not prove it (an empty
 * window, an outside node, or a failed coverage test), and cost the exact
 * search's scan-cost proxy (nodes scanned + cells visited + 20 per
 * certificate evaluation).  KC_ERR_ARG when n_nodes is not the resident
 * mesh's or the grid has more than 2e9 cells. */
int kc_grid_cell_stats(kc_ctx* ctx, long long n_nodes, const double* lon_branch, double cell_size, double lon_min,
                       double lat_min, int nx, int ny, int wrap, long long P, const double* lon, const double* lat,
                       int* nn, int* occ, double* cost, signed char* unprov, signed char* approx);

/* Digests of the Box-Muller draws over their whole input domain, for
 * checking the device arithmetic against the reference's: for every 32-bit
 * index j (u = (j + 1/2) 2^-32, the uniforms of diffusion.py:222-230) the
 * kick's r = sqrt(-2 log u), cos(2 pi u) and sin(2 pi u), summed as
 * mix(mix(j) ^ bits(value)) mod 2^64 (mix = one SplitMix64 round) into
 * out[0], out[1], out[2].  corrected = 0: the correctly rounded values;
 * 1: as kc_rng_normals and the kicks draw them (moved to the host C
 * library's value where its log / cos / sin round differently, so the draws
 * equal the reference's).  A check of _normal_pair
 * (src/kelp/numerics/diffusion.py:233-249) over all of its inputs. */
int kc_rng_domain_digests(kc_ctx* ctx, int corrected, unsigned long long* out);

/* Device error word since the last call: bit 0 an exact-search iteration cap
 * was hit, bit 1 kc_beach met a nearest_node outside [-n_nodes, n_nodes) and
 * left that particle unchanged. */
int kc_device_errors(kc_ctx* ctx, int* word);

/* Timing on the context's stream: record event `slot` (0..15), and the
 * elapsed milliseconds between two recorded events. */
int kc_event_record(kc_ctx* ctx, int slot);
int kc_event_elapsed(kc_ctx* ctx, int slot_a, int slot_b, float* ms);

/* Evict the L2 cache between timed steps: writes a library-owned buffer of
 * `bytes` (>= the 126 MB L2) on the context's stream. */
int kc_l2_flush(kc_ctx* ctx, long long bytes);

/* Page-locked host buffers for the end-to-end path. */
int kc_host_alloc(long long bytes, void** out);
int kc_host_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* KELP_CUDA_H */
