/* egg_b200 C-ABI: the B200 (sm_100a) structured TMOP smoother/untangler core.
 *
 * Plain C types only (pointers, sizes, ints, doubles); no exceptions cross the
 * boundary.  Every entry point returns an int status (EGG_B200_OK on success);
 * egg_b200_last_error() gives the message of the last failure on the calling
 * thread.  Each entry point names the reference interface it replaces
 * (file:line in the reference checkout).  All calls are synchronous: they
 * return after the session's CUDA stream has drained, like the reference's
 * q.wait() at every call boundary.
 */
#ifndef EGG_B200_H
#define EGG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EGG_B200_ABI_VERSION 1

/* Status codes.  EINVAL maps to Python ValueError, the others to RuntimeError
 * (the reference's std::invalid_argument / std::runtime_error split,
 * src/bindings.cpp:80-90,98-252,64-69). */
#define EGG_B200_OK 0
#define EGG_B200_EINVAL 1
#define EGG_B200_ERUNTIME 2
#define EGG_B200_ENODEV 3
#define EGG_B200_ENOTSUP 4

/* Objective kinds (src/metric.hpp:984-997 make_objective: "untangle",
 * "shape_size", anything else -> shape barrier). */
#define EGG_B200_OBJ_SHAPE 0
#define EGG_B200_OBJ_UNTANGLE 1
#define EGG_B200_OBJ_SHAPE_SIZE 2

/* Arithmetic of the sweep: plain fp64, or fp32 bulk with fp64 positions,
 * fp64 re-evaluation of near-degenerate samples and fp64 reductions. */
#define EGG_B200_PREC_FP64 0
#define EGG_B200_PREC_MIXED 1

/* Entity tags of constrained DOFs: the reference's frozen wire values
 * (src/entity_soa.hpp:37-56 EntityTag).  This core relaxes the entities
 * below; other tags are rejected with EGG_B200_ENOTSUP. */
#define EGG_B200_TAG_FREE 0
#define EGG_B200_TAG_LINESEG 1   /* record (sx, sy, ex, ey): segment, projection clamped to it */
#define EGG_B200_TAG_CIRCLE 2    /* record (cx, cy, r, -): radial projection */
#define EGG_B200_TAG_ELLIPSE 3   /* record (cx, cy, rx, ry): axis-aligned, radial-scaling projection */
#define EGG_B200_TAG_CIRCLEARC 6 /* record (cx, cy, r, t0, t1, closed): trimmed circular arc, angles in radians */
#define EGG_B200_TAG_ELLIPSEARC 7 /* record (cx, cy, a, b, phi, t0, t1, closed): rotated elliptic arc */
#define EGG_B200_TAG_QUADBEZIER 8 /* record (p0, p1, p2, t0, t1): quadratic Bezier, trimmed to [t0, t1] */
#define EGG_B200_TAG_CUBICBEZIER 9 /* record (p0, p1, p2, p3, t0, t1): cubic Bezier, trimmed to [t0, t1] */
#define EGG_B200_TAG_BSPLINE 10  /* record (degree, n_ctrl, t0, t1, closed, has_w, knots_at, ctrl_at, w_at):
                                  * B-spline / NURBS curve, degree <= 7; the *_at fields are offsets into
                                  * entity_arena (knots n_ctrl+degree+1, ctrl 2 n_ctrl, weights n_ctrl) */
#define EGG_B200_TAG_COMPOSITE 11 /* record (n_segs, rec_off, 0, 0, 0, 0, slice_at): a path of segment records
                                   * [tag, 12 params] at entity_arena[slice_at + rec_off ...]; segments are the
                                   * 2D curves (tags 1, 2, 3, 6, 7, 8, 9, 10, 15); a B-spline segment's blob
                                   * (degree, n_ctrl, knots, ctrl, t0, t1, w, has_w) offsets into the slice */
#define EGG_B200_TAG_LINERAIL 15 /* record (sx, sy, ex, ey): open-ended segment, released beyond its ends */
#define EGG_B200_TAG_SPHERE 4    /* 3D record (c(3), r, ax(3), ay(3)): untrimmed sphere, frame ax, ay, ax x ay */
#define EGG_B200_TAG_PLANE 5     /* 3D record (o(3), ax(3), ay(3)): untrimmed plane, orthonormal in-plane axes */
#define EGG_B200_TAG_CYLINDER 12 /* 3D record (o(3), ax(3), ay(3), r): untrimmed cylinder about ax x ay */
#define EGG_B200_TAG_LINE3 13    /* 3D record (p0(3), p1(3), t0, t1): line trimmed to [t0, t1] */
#define EGG_B200_TAG_LINERAIL3 16 /* 3D record (s(3), e(3)): open-ended segment, released beyond its ends */
#define EGG_B200_TAG_BSPLINESURF 14 /* 3D record (pu, pv, nu, nv, ku_at, kv_at, ctrl_at, w_at, has_w, trim_at):
                                     * B-spline / NURBS surface, degrees <= 7, the *_at fields offsets into
                                     * entity_arena (knots nu+pu+1 and nv+pv+1, ctrl 3 nu nv u-major, weights
                                     * nu nv); trim_at < 0 untrimmed, else the offset of (n_loop_entries,
                                     * loops_at, verts_at) describing the UV trim polygon */
#define EGG_B200_ENTITY_FIELDS 10 /* reals per entity record in entity_params */

typedef struct egg_b200_session egg_b200_session;

/* Everything the reference's session constructor takes, flattened:
 *   ctx_arrays (the "groups"/"energy_stencil" wire, egg/smoothing/flat_context.py:275-346)
 *   structured (egg/smoothing/cpp_backend.py:679-691)
 *   X0 (float64, global node order).
 * One merged group of moving DOFs, as the reference merges its groups
 * (src/sweep.hpp:729 build_merged_view).  Optional pointers may be NULL with
 * their length 0. */
typedef struct egg_b200_session_desc {
    int32_t dim;       /* 2 or 3 */
    int32_t precision; /* EGG_B200_PREC_* */
    int32_t device;    /* CUDA device ordinal, -1 = current */
    int32_t reserved0;

    int64_t num_nodes; /* M global nodes */
    const double* X;   /* [M*dim] */

    /* structured blocks */
    int32_t num_blocks;
    int32_t reserved1;
    const int32_t* interior_shapes;  /* [num_blocks*dim] */
    const int32_t* block_global_dof; /* concatenation of every block's row-major id array */
    int64_t num_halo;
    const int32_t* halo_src_block;  /* [num_halo] */
    const int32_t* halo_src_padded; /* [num_halo*dim] */
    const int32_t* halo_dst_block;  /* [num_halo] */
    const int32_t* halo_dst_padded; /* [num_halo*dim] */
    int64_t num_sing;
    const int32_t* sing_block;   /* [num_sing] */
    const int32_t* sing_logical; /* [num_sing*dim] */

    /* merged group of moving DOFs */
    int64_t ndof;
    const int32_t* dof_idx;          /* [ndof] global node id */
    const int32_t* P_of;             /* [ndof] stored occurrences per DOF */
    const int32_t* interior_block;   /* [ndof] or NULL; -1 = stored patch */
    const int32_t* interior_logical; /* [ndof*dim] or NULL */
    const int32_t* entity_tag;       /* [ndof] or NULL (all Free); EGG_B200_TAG_*, non-zero = constrained */
    int64_t total_samples;           /* sum(P_of) */
    const int32_t* gc;               /* [total_samples] */
    const int32_t* gn[3];            /* [total_samples] each, first dim used */
    const double* s[3];              /* [total_samples] each */
    const int32_t* role;             /* [total_samples] in [-1, dim] */
    const double* W_inv;             /* [dim*dim] (uniform) or [total_samples*dim*dim] */
    int64_t W_inv_len;
    const double* weight; /* NULL, [1] or [total_samples] */
    int64_t weight_len;

    /* energy stencil */
    int64_t es_num_samples;
    int32_t es_structured; /* 1: canonical cell stencil of the blocks, no index arrays */
    int32_t reserved2;
    const int32_t* es_gc;
    const int32_t* es_gn[3];
    const double* es_s[3];
    const double* es_W_inv; /* [dim*dim] or [es_num_samples*dim*dim] */
    int64_t es_W_inv_len;
    const double* es_weight; /* NULL, [1] or [es_num_samples] */
    int64_t es_weight_len;

    /* Entity record of every constrained DOF, EGG_B200_ENTITY_FIELDS reals
     * per DOF in group order (rows of Free DOFs are ignored): the DOF's row of
     * its entity partition's packed SoA records (src/entity_soa.hpp:98-108,
     * src/geometry.hpp:1760-1965 EntitySoA<E>::load), zero-padded.  NULL when
     * every DOF is Free.  A constrained DOF takes the reference's
     * boundary-kernel step (src/sweep.hpp:1286-1403): the Newton step reduced
     * onto the entity tangent, damped by omega before the line search, every
     * trial projected onto the entity.  A trimmed arc does so on the first
     * sweep of each run call; later sweeps search in its angle instead
     * (src/sweep.hpp:1718-1876). */
    const double* entity_params; /* [ndof * EGG_B200_ENTITY_FIELDS] or NULL */
    /* Variable-length entity data (B-spline knots, control points, weights),
     * addressed by offsets in the records.  A session with B-spline DOFs keeps
     * a per-DOF seed (the last foot parameter) for their iterative projection,
     * as the reference does (src/sweep.hpp:325-336): cold at creation and after
     * set_X / restore. */
    const double* entity_arena; /* [entity_arena_len] or NULL */
    int64_t entity_arena_len;

    /* Soft energy terms added to the shape objective (the group's curv_* and
     * dir_* tables and the energy stencil's dir_* table, src/bindings.cpp:
     * 380-410,471-480).  Per DOF in group order, K fixed slots each; a slot
     * of -1 pads.  Node ids are global.  Every moving DOF with a used slot
     * folds its terms into its Newton system and line search
     * (src/sweep.hpp:1307-1327,1461-1512,1600-1630, src/directional.hpp:
     * 221-279, src/curvature.hpp:113-183); reports add the whole-sample
     * directional total (src/sweep.hpp:1921, src/directional.hpp:281-299).
     * A curvature window is the 2D block-interface C2 term over four nodes;
     * a directional sample is kind 0 parallel (2 nodes), 1 line (3), 2 stem
     * (2); other kinds contribute nothing, as in the reference. */
    int32_t dir_k;             /* directional samples per DOF, 0 = none */
    int32_t curv_k;            /* curvature windows per DOF (2D), 0 = none */
    double dir_eps;            /* regularisation of the unit directions */
    const int32_t* dir_nodes;  /* [ndof*dir_k*4] */
    const int32_t* dir_slot;   /* [ndof*dir_k] the DOF's place in the sample */
    const int32_t* dir_kind;   /* [ndof*dir_k] */
    const double* dir_ref;     /* [ndof*dir_k*dim] frozen reference vector */
    const double* dir_weight;  /* [ndof*dir_k] */
    const int32_t* curv_nodes; /* [ndof*curv_k*4] */
    const int32_t* curv_slot;  /* [ndof*curv_k] */
    const double* curv_weight; /* [ndof*curv_k] */
    int64_t es_dir_num;        /* whole-sample directional table, 0 = none */
    double es_dir_eps;
    const int32_t* es_dir_nodes; /* [es_dir_num*4] */
    const int32_t* es_dir_kind;  /* [es_dir_num] */
    const double* es_dir_ref;    /* [es_dir_num*dim] */
    const double* es_dir_weight; /* [es_dir_num] */
} egg_b200_session_desc;

/* Control-net wire for one block (src/control_net.hpp:72-87 ControlNetHostT;
 * built by egg/smoothing/control_backend.py:76 build_control_wire): the
 * block's nodes are X = M C + b with M the tensor product of per-axis banded
 * clamped B-spline bases, node i of axis k reading controls off[k][i] ..
 * off[k][i] + k_supp - 1 with weights wt[k][i * k_supp + t].  Lattice and b
 * are row-major (last axis fastest) with the dim coordinates innermost. */
typedef struct egg_b200_control_desc {
    int32_t block;         /* block the net drives */
    int32_t k_supp;        /* support width per axis (degree + 1) */
    int32_t ctrl_shape[3]; /* controls per axis (first dim used) */
    int32_t reserved;
    int64_t off_len[3];    /* entries of off[k]: the block's node count on axis k */
    const int32_t* off[3]; /* first support control per node */
    const double* wt[3];   /* [off_len[k] * k_supp] basis weights */
    const double* C0;      /* [prod(ctrl_shape) * dim] initial lattice */
    int64_t n_free;
    const int32_t* free_idx; /* [n_free] flat lattice ids of the free controls */
    int64_t b_len;           /* prod(node counts) * dim */
    const double* b;         /* Boolean-sum boundary offset */
} egg_b200_control_desc;

/* Library / device. */
int egg_b200_abi_version(void);
const char* egg_b200_last_error(void);
int egg_b200_device_count(int* count);

/* Build a device-resident session: validate, re-home the global context onto
 * the packed per-block store and upload it once.
 * Replaces src/bindings.cpp:1153 make_structured_session and the
 * CppStructuredSweepSession constructor (src/bindings.cpp:1268-1281). */
int egg_b200_session_create(const egg_b200_session_desc* desc, egg_b200_session** out);

/* Batch session: n_meshes independent meshes (same dim, precision and
 * device) packed into one store, so every sweep is one launch per kernel
 * over all meshes and report chunks replay one captured CUDA graph.  Each
 * desc is validated against its own mesh.  The handle works with the
 * session calls above (run reports the sum over meshes and the global min;
 * get_X / set_X use the meshes' nodes concatenated in order, mesh m at
 * node_offsets[m]); run_fas is refused (ENOTSUP).  No counterpart in the
 * reference, whose sessions hold one mesh each (src/bindings.cpp:1268-1281);
 * a batch replaces n such sessions run one after another. */
int egg_b200_batch_create(const egg_b200_session_desc* descs, int32_t n_meshes, egg_b200_session** out);
/* Mesh count and, if node_offsets is not NULL, its n_meshes + 1 prefix
 * offsets into the concatenated global node order. */
int egg_b200_batch_size(egg_b200_session* s, int32_t* n_meshes, int64_t* node_offsets);
/* run with per-mesh reports: energies / mindets [report * n_meshes + mesh],
 * capacity and n_reported count reports (rows). */
int egg_b200_batch_run(egg_b200_session* s, int32_t n_sweeps, int32_t objective, double delta, double omega,
                       int32_t report_every, double* energies, double* mindets, int64_t capacity,
                       int64_t* n_reported);
/* One control net per mesh of a batch (desc[m].block is local to mesh m).
 * No counterpart in the reference (one net per session there). */
int egg_b200_batch_attach_controls(egg_b200_session* s, const egg_b200_control_desc* descs);
/* run_control on every mesh's net at once: kernels cover all nets, every
 * decision (convergence, step length, damping) is per mesh.  Outputs are
 * mesh-major with per-mesh stride n_outer + 1 (energies, mindets), n_outer
 * (alphas) and 8 * n_outer (pcg_*); counts is [n_meshes * 3]; iters and
 * converged are [n_meshes]. */
int egg_b200_batch_run_control(egg_b200_session* s, int32_t n_outer, int32_t objective, double grad_tol,
                               double alpha_min, double lm0, int32_t pcg_max_iter, double pcg_rtol,
                               int32_t pcg_forcing, double* energies, double* mindets, double* alphas,
                               double* pcg_iters, double* pcg_relres, int64_t* counts, int32_t* iters,
                               int32_t* converged);

/* Per-mesh energy and min det A of the resident state ([n_meshes] each). */
int egg_b200_batch_energy(egg_b200_session* s, int32_t objective, double delta, double* energies,
                          double* mindets);


/* Attach a control net to a session (the reference builds it inside the
 * session constructor, src/bindings.cpp:1234-1250 -> ControlSessionT,
 * src/control_solve.hpp:355).  Validation as src/bindings.cpp:507-556
 * (EINVAL).  ENOTSUP when the energy stencil is not the canonical cell
 * stencil of the blocks, or when a free control moves a node on a face the
 * block shares with another block. */
int egg_b200_session_attach_control(egg_b200_session* s, const egg_b200_control_desc* desc);

/* Damped reduced Gauss-Newton on the free controls with Jacobi-preconditioned
 * matrix-free PCG (src/control_solve.hpp:533-700 run_plain, :761 pcg_solve;
 * binding src/bindings.cpp:1382-1437 run_control).  Shape objectives only
 * (untangle -> EINVAL); EINVAL without a control net.  Outputs (capacities in
 * parentheses): energies and mindets (n_outer + 1, the initial state first),
 * alphas (n_outer), pcg_iters and pcg_relres (8 * n_outer, one per PCG
 * solve); counts[0..2] = entries written to energies, alphas, pcg_*. */
int egg_b200_session_run_control(egg_b200_session* s, int32_t n_outer, int32_t objective, double grad_tol,
                                 double alpha_min, double lm0, int32_t pcg_max_iter, double pcg_rtol,
                                 int32_t pcg_forcing, double* energies, double* mindets, double* alphas,
                                 double* pcg_iters, double* pcg_relres, int64_t* counts, int32_t* iters,
                                 int32_t* converged);

/* One wall face of a single control net (src/control_net.hpp
 * ControlWallHost; wire src/bindings.cpp:557-590, built by
 * egg/smoothing/control_backend.py:137-175 from
 * egg/smoothing/control_wall.py WallSpec): the net's face `axis`/`side`
 * lies on a codim-1 entity (a 2D curve or a 3D surface with a fixed-size
 * record: tags 1-3, 6-9, 15 in 2D; 4, 5, 12 in 3D).  Leg j pairs the
 * wall-row control p0[j], which slides on the entity, with its inward
 * neighbour p1[j]; mode 0 leaves p1 free, 1 adds the penalty
 * weight[j] / |leg|^2 on the leg's tangential components, 2 holds p1 on the
 * wall normal through p0 (one height unknown). */
typedef struct egg_b200_control_wall {
    int32_t axis, side, mode, tag;
    int64_t n_legs;
    const int32_t* p0;     /* [n_legs] lattice ids (free controls) */
    const int32_t* p1;     /* [n_legs] */
    const double* weight;  /* [n_legs] */
    const double* params;  /* entity record, params_len <= EGG_B200_ENTITY_FIELDS reals */
    int64_t params_len;
} egg_b200_control_wall;

/* Attach a control net with walls (the reference builds it inside the
 * session constructor when the control wire carries "walls": ControlSessionT
 * with init_walls, src/control_solve.hpp:498,828).  X0 [node count * dim] is
 * the block's exact node field; its non-wall boundary rows anchor the
 * Boolean-sum re-extension.  egg_b200_session_run_control then rebuilds the
 * wall frame before every outer iteration and once at the end
 * (src/control_solve.hpp:1331 run_walls).  EINVAL on the reference's
 * validation failures; ENOTSUP for segmented wall entities (B-spline,
 * composite), which the reference's wire builder refuses too. */
int egg_b200_session_attach_control_walls(egg_b200_session* s, const egg_b200_control_desc* desc, const double* X0,
                                          int64_t X0_len, int32_t n_walls, const egg_b200_control_wall* walls);

/* Multi-block control topology wire (src/control_net.hpp ControlTopoHostT;
 * src/bindings.cpp:596-690 unpack_control_topo; built by
 * egg/smoothing/control_backend.py run_control_topo): one net per block,
 * stacked in wire order (nets[i].C0, free_idx and n_free are ignored: every
 * control is free and C0 is the stacked lattice), the reduction CSR dC = R dq
 * over the nsd = total controls * dim stacked components (r_off has nsd + 1
 * entries, columns < nq), and optional penalty rows 1/2 sum_j w_j (P_j C)^2
 * (p_off_len == 0 for none; columns < nsd), and optionally the
 * sliding-wall frames (egg_b200_control_slide): run_control then rebuilds
 * the frame before every outer iteration and once at the end
 * (src/control_solve.hpp:2771 rebuild_frame) and reports each rebuild's
 * energy jump. */
/* Sliding-wall frames of a topology (src/control_net.hpp ControlTopoHostT
 * slide / wall_faces / seam_face; wire built by
 * egg/smoothing/control_backend.py:472-560 _attach_slide_wire).  A sliding
 * root is a reduced unknown riding an entity: its representative stacked
 * control rep_row is projected every outer iteration, the tangent frame at
 * the foot rewrites the reduction entries r_entry[e] = base[e] *
 * t[kt[e]][comp[e]], and every member row moves by member_coef * (foot -
 * rep).  Entity records are the reference's decode blobs: the fixed-size
 * records of the constrained-boundary tags, a 2D B-spline curve as
 * (degree, n_ctrl, knot_off, ctrl_off, t0, t1, w_off, has_w) and a 2D
 * composite path as (n_segs, rec_off), offsets into `arena`. */
typedef struct egg_b200_control_slide {
    int32_t rep_row, tag;
    int64_t n_members;
    const int32_t* members;     /* [n_members] stacked control rows */
    const double* member_coef;  /* [n_members] */
    const double* params;       /* entity blob, params_len reals */
    int64_t params_len;
    int64_t n_entries;
    const int32_t* r_entry;     /* [n_entries] reduction CSR entries */
    const int32_t* comp;        /* [n_entries] component 0..dim-1 */
    const int32_t* kt;          /* [n_entries] tangent slot 0..dim-2 */
    const double* base;         /* [n_entries] frame-free coefficient */
} egg_b200_control_slide;

/* A wall face of a net: its nodes on `axis`/`side` are re-extended against
 * the entity's projection of the spline every frame. */
typedef struct egg_b200_control_wall_face {
    int32_t net, axis, side, tag;
    const double* params; /* entity blob */
    int64_t params_len;
} egg_b200_control_wall_face;

typedef struct egg_b200_control_topo_desc {
    int32_t n_nets;
    int32_t reserved;
    const egg_b200_control_desc* nets; /* [n_nets] */
    const double* C0;                  /* [C0_len = total controls * dim] */
    int64_t C0_len;
    int64_t nq;
    const int32_t* r_off;
    int64_t r_off_len;
    const int32_t* r_col;
    const double* r_coef;
    int64_t r_nnz;
    const int32_t* p_off;
    int64_t p_off_len;
    const int32_t* p_col;
    const double* p_coef;
    int64_t p_nnz;
    const double* p_w;
    int64_t p_w_len;
    /* sliding-wall frames (n_slide == 0: none; the rest is then unread) */
    int32_t n_slide;
    int32_t n_wall_faces;
    const egg_b200_control_slide* slide;          /* [n_slide] */
    const egg_b200_control_wall_face* wall_faces; /* [n_wall_faces] */
    const int32_t* seam_face; /* [n_nets * 2 * dim]: face (axis, side) of each net lies on a seam */
    const double* X0;         /* every net's exact node field, concatenated in net order */
    int64_t X0_len;
    const double* arena;      /* variable-length entity payloads */
    int64_t arena_len;
} egg_b200_control_topo_desc;

/* Attach a multi-block control topology (the reference builds it inside the
 * session constructor when control['blocks'] is present, src/bindings.cpp:
 * 1181-1235 -> ControlTopoSessionT, src/control_solve.hpp:1585).  The alias
 * groups of shared nodes come from the session's own owner / copy tables.
 * Validation messages as the reference's ("control topo: ...", EINVAL);
 * ENOTSUP when a block carries no net or the energy stencil is not the
 * canonical cell stencil of the blocks.  X is left as it is (a run, set_C or
 * set_control_b evaluates X = M C + b and refreshes the copies).
 * egg_b200_session_run_control then runs the topology's single
 * reduced problem (one report); get_C / set_C use the stacked lattice. */
int egg_b200_session_attach_control_topo(egg_b200_session* s, const egg_b200_control_topo_desc* desc);
/* Replace the reduction CSR (src/control_solve.hpp:2057 set_reduction;
 * binding src/bindings.cpp:1474-1495 set_control_reduction). */
int egg_b200_session_set_control_reduction(egg_b200_session* s, int64_t nq, const int32_t* off, int64_t off_len,
                                           const int32_t* col, const double* coef, int64_t nnz);
/* Replace the penalty rows; off_len == 0 removes them (src/control_solve.hpp:
 * 2120 set_penalty; binding src/bindings.cpp:1497-1516). */
int egg_b200_session_set_control_penalty(egg_b200_session* s, const int32_t* off, int64_t off_len,
                                         const int32_t* col, const double* coef, int64_t nnz, const double* w,
                                         int64_t w_len);
/* Replace net `net_index`'s Boolean-sum offset b (node count * dim reals) and
 * re-evaluate X (src/control_solve.hpp:2172 set_b; binding
 * src/bindings.cpp:1518-1530 set_control_b). */
int egg_b200_session_set_control_b(egg_b200_session* s, int32_t net_index, const double* b, int64_t len);

/* egg_b200_session_run_control with the options of the reference's full
 * ControlOptions (src/control_solve.hpp:308-330): model_db switches the
 * db/dC linearisation of a topology's sliding-wall frames, and frame_jumps
 * (capacity n_outer) receives the energy jump of each frame rebuild
 * (*n_frame_jumps entries; none without sliding-wall frames). */
int egg_b200_session_run_control_ex(egg_b200_session* s, int32_t n_outer, int32_t objective, double grad_tol,
                                    double alpha_min, double lm0, int32_t pcg_max_iter, double pcg_rtol,
                                    int32_t pcg_forcing, int32_t model_db, double* energies, double* mindets,
                                    double* alphas, double* pcg_iters, double* pcg_relres, int64_t* counts,
                                    int32_t* iters, int32_t* converged, double* frame_jumps, int64_t* n_frame_jumps);

/* The resident control lattice (prod(ctrl_shape) * dim reals; stacked over
 * the meshes of a batch or the nets of a topology): size, download, and
 * upload followed by the evaluation X = M C + b into the store
 * (src/bindings.cpp:1441-1480). */
int egg_b200_session_control_size(egg_b200_session* s, int64_t* n_reals);
int egg_b200_session_get_C(egg_b200_session* s, double* C, int64_t len);
int egg_b200_session_set_C(egg_b200_session* s, const double* C, int64_t len);

/* Release every device allocation of the session (RAII end of the reference
 * session, src/device.hpp:51). */
int egg_b200_session_destroy(egg_b200_session* s);

/* n_sweeps of double-buffered block-Jacobi on the resident store; writes
 * ceil(n/k) (k = report_every, or 1 report when report_every <= 0) energies
 * and min-dets.  Replaces CppStructuredSweepSession::run
 * (src/bindings.cpp:1292-1304) -> run_block_jacobi (src/sweep.hpp:2027). */
int egg_b200_session_run(egg_b200_session* s, int32_t n_sweeps, int32_t objective, double delta,
                         double omega, int32_t report_every, double* energies, double* mindets,
                         int64_t capacity, int64_t* n_reported);

/* n_cycles FAS V-cycles (nu_pre / nu_post Jacobi sweeps per level, at most
 * nu_coarse on the coarsest level, the hierarchy clipped to max_levels levels
 * including the fine one) on the resident store; writes one energy / min det
 * per cycle.  Shape objectives only (untangle -> EINVAL).  Falls back to
 * n_cycles*(nu_pre+nu_post) Jacobi sweeps reported every nu_pre+nu_post when
 * no coarse level exists.  Replaces CppStructuredSweepSession::run_fas
 * (src/bindings.cpp:1311-1335) -> egg::run_fas (src/fas.hpp:398). */
int egg_b200_session_run_fas(egg_b200_session* s, int32_t n_cycles, int32_t nu_pre, int32_t nu_post,
                             int32_t nu_coarse, double omega, int32_t max_levels, int32_t objective,
                             double* energies, double* mindets, int64_t capacity, int64_t* n_reported);

/* Coarse hierarchy: number of coarse levels, and for level `level` (0 =
 * first coarse level) each block's interior shape [num_blocks * dim].
 * Replaces CppStructuredSweepSession::mg_levels (src/bindings.cpp:1339-1356). */
int egg_b200_session_mg_levels(egg_b200_session* s, int32_t* n_levels);
int egg_b200_session_mg_level_shapes(egg_b200_session* s, int32_t level, int32_t* shapes, int64_t len);

/* Energy and min det A of the resident state under an objective (the
 * reduction of src/sweep.hpp:1881 reduce_energy_mindet, without a sweep). */
int egg_b200_session_energy(egg_b200_session* s, int32_t objective, double delta, double* energy,
                            double* mindet);

/* The same energy and min det A through a variant that allocates nothing:
 * the reduction's per-CTA partials and its two results live in one
 * file-scope __device__ array of 3 * EGG_B200_NOALLOC_MAX_PARTIALS + 2
 * doubles (96 KiB + 16 B per device) instead of session buffers, and the
 * call makes no cudaMalloc, cudaFree or other allocating library call on
 * its success path (a failure stores its message like every other entry
 * point).  n_partials is the number of reduction CTAs: 0 picks the
 * session's own count, which gives results bit-identical to
 * egg_b200_session_energy; 1..EGG_B200_NOALLOC_MAX_PARTIALS sets it; larger
 * or negative values fail with EGG_B200_EINVAL.  Every call on a device
 * shares the one array: calls whose GPU work overlaps (concurrent host
 * threads, or sessions on different streams) race on it.  Each call
 * returns only after its own result has reached the host.  The first call
 * on a device looks up the array's device address and keeps it for the
 * process; after cudaDeviceReset that address is stale, so a process that
 * resets a device must not call this entry point on it again.
 * No counterpart in the reference: it exists for callers that must not
 * allocate device memory per call. */
#define EGG_B200_NOALLOC_MAX_PARTIALS 4096
int egg_b200_session_energy_noalloc(egg_b200_session* s, int32_t objective, double delta,
                                    int32_t n_partials, double* energy, double* mindet);

/* Page-locked host buffers from a process-wide pool (no counterpart in the
 * reference).  get_X into such a buffer is one DMA, with no staging copy.
 * acquire returns EGG_B200_ERUNTIME when the page-lock fails; the caller
 * then uses ordinary memory.  release takes a pointer that acquire returned
 * (anything else fails with EGG_B200_EINVAL) and returns it to the pool; the
 * pool keeps at most two idle buffers per size and 1 GiB of idle buffers in
 * all, and frees the rest.  trim frees every idle buffer and returns the
 * bytes it freed. */
int egg_b200_pinned_acquire(int64_t bytes, void** out);
int egg_b200_pinned_release(void* p);
int64_t egg_b200_pinned_trim(void);

/* Download the resident positions in GLOBAL node order ([num_nodes*dim]).
 * Replaces CppStructuredSweepSession::get_X (src/bindings.cpp:1359-1376). */
int egg_b200_session_get_X(egg_b200_session* s, double* X, int64_t len);

/* Upload positions in global node order, scattered into every copy.
 * Replaces SweepDeviceContextT::upload_X (src/sweep.hpp:552-557). */
int egg_b200_session_set_X(egg_b200_session* s, const double* X, int64_t len);

/* Session facts: [0] dim, [1] global nodes, [2] packed store nodes, [3] moving
 * DOFs, [4] structured-interior DOFs, [5] stored-patch DOFs, [6] owner->copy
 * entries, [7] energy samples, [8] structured energy stencil (0/1),
 * [9] precision, [10] vertex Newton updates issued since creation or the
 * last reset_stats (every DOF relaxed once, at any FAS level). */
int egg_b200_session_info(egg_b200_session* s, int64_t* out, int32_t n);

/* Per-kernel CUDA-event timing on the session stream (off by default).
 * kernel ids: 0 interior sweep, 1 stored-patch sweep, 2 owner->copy broadcast,
 * 3 energy reduction, 4 reduction finalize, 5 buffer copy, 6 FAS transfers,
 * 7 control-net kernels. */
int egg_b200_session_set_profiling(egg_b200_session* s, int32_t enable);
int egg_b200_session_kernel_stats(egg_b200_session* s, int32_t kernel_id, double* total_ms,
                                  int64_t* launches);
int egg_b200_session_reset_stats(egg_b200_session* s);

/* Device-side checkpoint of the resident positions (one extra store-sized
 * buffer) and restore from it; no host traffic.  The reference has no solver
 * checkpoint (sessions are resumed by get_X/set_X, src/bindings.cpp:1359);
 * this is the device-resident form of that round trip. */
int egg_b200_session_checkpoint(egg_b200_session* s);
int egg_b200_session_restore(egg_b200_session* s);

/* Autotuner of the interior sweep kernel: times each launch variant (cells
 * per CTA, resident CTAs per SM) on the session's own resident data without
 * changing it, keeps the fastest and returns its index.  Runs automatically
 * before the first sweep unless EGG_B200_AUTOTUNE=0.  No counterpart in the
 * reference (AdaptiveCpp picks launch shapes itself). */
int egg_b200_session_autotune(egg_b200_session* s, int32_t objective, int32_t reps, int32_t* chosen);
int egg_b200_session_set_variant(egg_b200_session* s, int32_t variant);
/* Current variant, per-variant shape (ci, cj, ck, min CTAs/SM, full_dof)
 * [5*n] -- 2D: cells per CTA, or DOFs per CTA when full_dof = 1; 3D: DOFs per
 * CTA -- and the tuned times in ms [n], for the first n <=
 * EGG_B200_NUM_VARIANTS variants. */
#define EGG_B200_NUM_VARIANTS 5
int egg_b200_session_variant_info(egg_b200_session* s, int32_t* variant, int32_t* shape, double* times_ms,
                                  int32_t n);

/* Kernel launches issued by the session since creation or the last
 * reset_stats (every kernel of this library counts, copies excluded). */
int egg_b200_session_launch_count(egg_b200_session* s, int64_t* launches);

/* The session's CUDA stream (a cudaStream_t), on which every kernel and copy
 * of the session is issued, so that a host can record its own events around
 * a call.  Session-specific instrumentation (the reference queue is
 * internal). */
int egg_b200_session_stream(egg_b200_session* s, void** stream);

/* Device evaluation of the per-sample metric on n vec(T) rows (the GPU twin of
 * the reference's oracle binding metric_eval, src/bindings.cpp:1778-1800):
 * t [n*4] -> mu [n], grad [n*4], hess [n*16]. */
int egg_b200_metric_eval(int32_t objective, double delta, const double* t, int64_t n, double* mu,
                         double* grad, double* hess);

/* Device evaluation of the 3D metric along the kernels' own code path: for n
 * rows of vec(T) [9] and directions v [3]: mu [n], the gradient over vec(T)
 * [9n] and the contracted Hessian sum_cc' v_c v_c' H[(i,c),(j,c')] packed
 * (xx, xy, xz, yy, yz, zz) [6n].  GPU twin of the oracle binding
 * metric_eval_3d (src/bindings.cpp:1806-1815). */
int egg_b200_metric3_probe(int32_t objective, double delta, const double* t, const double* v, int64_t n,
                           double* mu, double* grad9, double* hv);

/* Device evaluation of one stored patch (grad, hess, energy, mindet) and its
 * Newton step (the GPU twin of the oracle bindings patch_eval / newton_step,
 * src/bindings.cpp:1858-2005).  X [n_nodes*2]; per occurrence gc, gn0, gn1,
 * s0, s1, W_inv [P*4], role.  out: grad[2], hess[4], energy, mindet, step[2]. */
int egg_b200_patch_eval(int32_t objective, double delta, const double* X, int64_t n_nodes,
                        int32_t P, const int32_t* gc, const int32_t* gn0, const int32_t* gn1,
                        const double* s0, const double* s1, const double* W_inv,
                        const int32_t* role, double* grad, double* hess, double* energy,
                        double* mindet, double* step);

/* Free-DOF Newton step -H^{-1} g with the zero-gradient and non-finite
 * fallbacks, evaluated on the device (the oracle binding newton_step,
 * src/bindings.cpp:2100-2130, for the Free tag). grad[2], hess[4] -> step[2]. */
int egg_b200_newton_step(const double* grad, const double* hess, double* step);

/* Constrained-DOF Newton step and projection, evaluated on the device (the
 * oracle binding newton_step, src/bindings.cpp:2103-2130, for an entity tag;
 * src/patch.hpp:396-413 newton_delta): step = the Newton step reduced onto the
 * entity tangent at pos (a rail released beyond its ends takes the full step),
 * foot = the projection of pos onto the entity.  tag is one of the
 * EGG_B200_TAG_* curves; record holds its EGG_B200_ENTITY_FIELDS reals.
 * grad[2], hess[4] (row-major), pos[2] -> step[2], foot[2]. */
int egg_b200_entity_step(int32_t tag, const double* record, const double* grad, const double* hess,
                         const double* pos, double* step, double* foot);

/* Projection of n points onto one constrained-boundary entity, with the
 * orthonormal tangent basis at each foot, evaluated on the device (the GPU
 * twin of the reference's oracle bindings geometry_project_batch,
 * src/bindings.cpp:1891-1990, and -- for a 2D curve and n = 1 --
 * geometry_project / geometry_tangent, src/bindings.cpp:1859-1889).
 * dim 2: a curve tag, basis [n*2] (the unit tangent at the foot); dim 3: a
 * surface (Plane, Sphere, Cylinder: basis [n*3*2]) or a line (Line3,
 * LineRail3: basis [n*3]), packed (point, component, column).  record holds
 * EGG_B200_ENTITY_FIELDS reals as in entity_params; B-spline and composite
 * records address `arena` by offset.  q [n*dim] -> foot [n*dim]. */
int egg_b200_entity_frame(int32_t dim, int32_t tag, const double* record, const double* arena, int64_t arena_len,
                          const double* q, int64_t n, double* foot, double* basis);

/* Directional soft-term total and its gradient over a sample table,
 * evaluated on the device (the GPU twin of the oracle binding
 * directional_eval, src/bindings.cpp:1819-1857).  X [n_nodes*dim]; per
 * sample nodes [4] (-1 pads), kind (parallel 0, line 1, stem 2), ref [dim],
 * weight.  Out: energy, grad [n_nodes*dim]. */
int egg_b200_directional_eval(int32_t dim, const double* X, int64_t n_nodes, int64_t n, const int32_t* nodes,
                              const int32_t* kind, const double* ref, const double* weight, double eps,
                              double* energy, double* grad);

/* Device-side wire build: the bulk index arrays of the sweep-context wire,
 * computed by kernels from the blocks' global node ids.  Replaces the array
 * work of egg/smoothing/flat_context.py:136-346 (build_flat_context, with
 * its cell_stencil at :40-121); the per-entity partitions, soft-term tables
 * and W_inv rows stay with the host caller.  Outputs equal the reference
 * builder's bit for bit:
 *   group: dof_idx, P_of, interior_block, interior_logical [n_dofs*dim],
 *          role, gc, gn0..gn{dim-1} (int32) and s0..s{dim-1} (float64) [n_rows];
 *   energy stencil (energy_arrays != 0): gc, gn*, s* [n_samples].
 * moving[n] = 1 marks a moving DOF (Free or constrained); stored[n] = 1
 * (optional) forces a stored patch (constrained DOFs; their interior_logical
 * is still filled, interior_block is -1).  synth_interior = 1 when the target
 * is a uniform multiple of the identity: interior-eligible DOFs then carry no
 * rows.  Node ids must lie in [0, num_nodes) (EGG_B200_EINVAL otherwise) and
 * fit int32 (EGG_B200_ENOTSUP).  device < 0 uses the current device.
 * build keeps the arrays on the device; sizes gives {n_dofs, n_rows,
 * n_samples}; download copies every non-NULL output (host memory sized from
 * sizes); destroy frees them. */
typedef struct egg_b200_wire egg_b200_wire;
typedef struct egg_b200_wire_desc {
    int32_t dim;
    int32_t num_blocks;
    const int32_t* shapes;    /* [num_blocks * dim] nodes per axis */
    const int64_t* block_ids; /* global ids of every block's nodes, C order, blocks back to back */
    int64_t num_nodes;
    const uint8_t* moving;    /* [num_nodes] */
    const uint8_t* stored;    /* [num_nodes] or NULL */
    int32_t synth_interior;
    int32_t energy_arrays;
    int32_t device;
} egg_b200_wire_desc;
typedef struct egg_b200_wire_out {
    int32_t* dof_idx;
    int32_t* P_of;
    int32_t* interior_block;
    int32_t* interior_logical;
    int32_t* role;
    int64_t* sid;             /* [n_rows] sample id of each row (2^dim * cell + corner) */
    int32_t* gc;
    int32_t* gn[3];
    double* s[3];
    int32_t* es_gc;
    int32_t* es_gn[3];
    double* es_s[3];
} egg_b200_wire_out;
int egg_b200_wire_build(const egg_b200_wire_desc* desc, egg_b200_wire** out);
int egg_b200_wire_sizes(egg_b200_wire* w, int64_t* sizes);
int egg_b200_wire_download(egg_b200_wire* w, const egg_b200_wire_out* out);
int egg_b200_wire_destroy(egg_b200_wire* w);

#ifdef __cplusplus
}
#endif

#endif /* EGG_B200_H */
