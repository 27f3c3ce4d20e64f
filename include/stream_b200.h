/*
 * stream_b200 C ABI: the drop-in boundary for the PFEM remesh-and-solve path.
 *
 * One shared library (libstream_b200.so, aliased as libmesh.so, libnumerics.so
 * and libgeometry.so) exports every function below.  Names, argument order and
 * meaning of the first group in each section are those of the reference's
 * extern "C" blocks (cited per function); "additive" entry points are new and
 * return an int status (0 = ok, otherwise a bitmask of STREAM_ST_*).
 *
 * Conventions shared with the reference: opaque handles created/destroyed by
 * the caller; input arrays are copied on set; outputs go to caller-allocated
 * host buffers sized by a prior size query; point ids in outputs are in Morton
 * order (see AlphaShape3D_get_permutation).  Reference entry points that
 * return void record failures in the handle (AlphaShape3D_get_status) and in
 * stream_b200_last_error(); no C++ exception crosses this boundary.  Calls on
 * distinct handles are independent (each handle owns a CUDA stream); a handle
 * must not be used by two host threads at once.
 */
#ifndef STREAM_B200_H
#define STREAM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status bits (int return values and AlphaShape3D_get_status). */
#define STREAM_ST_STACK_OVERFLOW   0x001 /* BVH traversal stack exhausted */
#define STREAM_ST_WALK_CAP         0x002 /* 3D: cavity walk hit its 100-step cap (reference behaviour, informational);
                                            Mesh2D: a star ran out of queries or LBVH visits */
#define STREAM_ST_BROKEN_CYCLE     0x004 /* cavity boundary cycle not closed */
#define STREAM_ST_TET_CAP          0x008 /* local tet list overflow (Mesh2D: a star ran out of local ids) */
#define STREAM_ST_EXACT_OVERFLOW   0x010 /* exact expansion longer than its buffer */
#define STREAM_ST_LOOKBACK_TIMEOUT 0x020 /* decoupled look-back gave up (sort/scan) */
#define STREAM_ST_TRUNCATED        0x040 /* a star had > 124 candidates (reference behaviour, informational) */
#define STREAM_ST_BAD_INPUT        0x080 /* invalid argument */
#define STREAM_ST_CUDA_ERROR       0x100 /* CUDA runtime failure */
#define STREAM_ST_INCOMPLETE       0x200 /* Mesh2D: a star still unverified after Mesh2D_insert_iterative */

/* ------------------------------------------------------------ library --- */
/* Message of the last failure seen by the calling thread ("" if none). */
const char* stream_b200_last_error(void);
/* 1 when a compute-capability 10.0 GPU is visible. */
int stream_b200_device_ok(void);
/* Kernel launches issued by the library since it was loaded. */
unsigned long long stream_b200_launch_count(void);

/* ---------------------------------------------------------- AlphaShape3D ---
 * Reference: include/mesh/DirectAlphaShape3D.hpp:40-69 (declarations; its
 * AlphaShape2D_set_nodes at :52 is a typo for the AlphaShape3D_set_nodes that
 * src/mesh/DirectAlphaShape3D.cpp:764 defines) and
 * src/mesh/DirectAlphaShape3D.cpp:754-810 (definitions). */
typedef struct AlphaShape3D AlphaShape3D;

/* DirectAlphaShape3D.cpp:757-759 */
AlphaShape3D* AlphaShape3D_create(void);
/* DirectAlphaShape3D.cpp:761-763 */
void AlphaShape3D_destroy(AlphaShape3D* ashape);
/* DirectAlphaShape3D.cpp:764-777: coords nnodes x 3 row-major, alpha nnodes. */
void AlphaShape3D_set_nodes(AlphaShape3D* ashape, uint32_t nnodes, const float* coords, const float* alpha);
/* DirectAlphaShape3D.cpp:780-782: LBVH build + candidate-neighbour pass. */
void AlphaShape3D_init(AlphaShape3D* ashape);
/* DirectAlphaShape3D.cpp:785-788: star Delaunay, alpha filter, compress. */
void AlphaShape3D_compute(AlphaShape3D* ashape);
/* DirectAlphaShape3D.cpp:791-793 */
uint32_t AlphaShape3D_get_nelem(const AlphaShape3D* ashape);
/* DirectAlphaShape3D.cpp:796-800: elems is nelem x 4 (Morton ids; a = owner). */
void AlphaShape3D_get_elem(const AlphaShape3D* ashape, uint32_t* elems);
/* DirectAlphaShape3D.cpp:802-810: nodes is nnodes x 3, Morton order. */
void AlphaShape3D_get_ordered_nodes(AlphaShape3D* ashape, float* nodes);

/* Additive.  Morton code width of the LBVH: 63 (reference) or 30. */
int AlphaShape3D_set_morton_bits(AlphaShape3D* ashape, int bits);
/* Additive.  Device input: d_xyza is nnodes float4 (x, y, z, alpha) in GPU memory. */
int AlphaShape3D_set_nodes_device(AlphaShape3D* ashape, uint32_t nnodes, const float* d_xyza);
/* Additive.  Status bits of the last call on this handle. */
int AlphaShape3D_get_status(const AlphaShape3D* ashape);
/* Additive.  out4 = {status, deferred stars, truncated stars, exact-stage calls}. */
int AlphaShape3D_get_counters(const AlphaShape3D* ashape, uint32_t* out4);
/* Additive (C++-only getPermutation in the reference, DirectAlphaShape3D.cpp:75-80):
 * perm[i] = input index of Morton-ordered point i.  Returns nnodes. */
uint32_t AlphaShape3D_get_permutation(const AlphaShape3D* ashape, uint32_t* perm);
/* Additive (C++-only getEdge, DirectAlphaShape3D.cpp:90-98). */
uint32_t AlphaShape3D_get_nedge(const AlphaShape3D* ashape);
/* row nnodes+1, neig nedge, edge_is_bnd nedge (1 = used by <= 3 kept tets).  Returns nedge. */
uint32_t AlphaShape3D_get_edges(const AlphaShape3D* ashape, uint32_t* row, uint32_t* neig, uint8_t* edge_is_bnd);
/* Additive (C++-only getBoundaryNodes, DirectAlphaShape3D.cpp:101-105): free-surface flags. */
uint32_t AlphaShape3D_get_boundary_nodes(const AlphaShape3D* ashape, uint8_t* is_bnd);
/* Additive diagnostics: nineig n, nkeep n, cand n x 124 (traversal order). */
int AlphaShape3D_get_stars(const AlphaShape3D* ashape, uint32_t* nineig, uint8_t* nkeep, uint32_t* cand);
/* Additive: device pointers of the resident outputs (valid until the next set/init/compute). */
int AlphaShape3D_get_device_outputs(const AlphaShape3D* ashape, const void** obj_m, const void** elems,
                                    const void** row, const void** neig, const void** node_is_bnd);
/* Additive: per-stage device timing of init()+compute() (CUDA events). */
int AlphaShape3D_set_profiling(AlphaShape3D* ashape, int on);
/* ms8 = {bbox+Morton, radix sort, gather+Karras+fit, candidates, star, star exact
 * stage, scans + size read-back, compress} of the last init()+compute(). */
int AlphaShape3D_get_profile(AlphaShape3D* ashape, float* ms8);
/* The same stages into ms (at most count values; *written = how many, may be
 * NULL), for callers that size the array from the returned count. */
int AlphaShape3D_get_profile_stages(AlphaShape3D* ashape, float* ms, uint32_t count, uint32_t* written);
/* Additive: work counters for roofline accounting.  With set_work_counters(1)
 * compute() runs the fast star pass in a counting build (same decisions and
 * outputs) and get_work reports out2 = {stage-1 FP32 insphere tests, stage-2
 * FP64 filter evaluations}, 117 floating-point operations each. */
int AlphaShape3D_set_work_counters(AlphaShape3D* ashape, int on);
int AlphaShape3D_get_work(AlphaShape3D* ashape, uint64_t* out2);
/* Additive: run this handle's work on a caller-owned cudaStream_t (NULL: the
 * handle's own stream again).  Pending work is synchronised first. */
int AlphaShape3D_set_stream(AlphaShape3D* ashape, void* stream);
/* Additive: wait for the handle's stream. */
int AlphaShape3D_synchronize(AlphaShape3D* ashape);
/* Additive test entry: the star kernel's conflict decision for m quintuples
 * (pts m x 5 x 3, ids m x 5) -> out[m], the reference's 'det'
 * (DirectAlphaShape3D.cpp:423-480). */
int stream_b200_conflict_batch(uint32_t m, const float* pts, const uint32_t* ids, float* out);
/* No counterpart in the reference.  The same decisions as
 * stream_b200_conflict_batch for callers that cannot allocate device memory
 * (a host that only hands over device buffers it already owns and forbids new
 * allocations, or a plugin inside such a host): d_pts (m x 5 x 3), d_ids
 * (m x 5) and d_out (m) are device arrays the caller provides, and the exact
 * stage's scratch lives in a fixed 3.3 MiB device array created with the
 * library in every GPU that loads it.  At most 256 quintuples per call (more
 * is rejected with STREAM_ST_BAD_INPUT).  No cudaMalloc or cudaFree.  The first
 * call on a device looks up that array's device address (cudaGetSymbolAddress)
 * and caches it, so make it before any stream capture; after cudaDeviceReset
 * on that device, do not call it again in the same process.  All calls share
 * the array: calls whose work overlaps on the GPU race and must not be issued.
 * stream may be NULL; the call waits for its work and returns the status bits
 * (0 = ok). */
int stream_b200_conflict_batch_noalloc(uint32_t m, const float* d_pts, const uint32_t* d_ids, float* d_out,
                                       void* stream);

/* ---------------------------------------------------------- AlphaShape2D ---
 * Reference: include/mesh/DirectAlphaShape2D.hpp:48-67 (declarations) and
 * src/mesh/DirectAlphaShape2D.cpp:698-753 (definitions).  Output ids are Morton
 * ordered (AlphaShape2D_get_permutation maps them back). */
typedef struct AlphaShape2D AlphaShape2D;

/* DirectAlphaShape2D.cpp:698-700 */
AlphaShape2D* AlphaShape2D_create(void);
/* DirectAlphaShape2D.cpp:702-704 */
void AlphaShape2D_destroy(AlphaShape2D* ashape);
/* DirectAlphaShape2D.cpp:708-721: coords nnodes x 2 row-major, alpha nnodes. */
void AlphaShape2D_set_nodes(AlphaShape2D* ashape, uint32_t nnodes, const float* coords, const float* alpha);
/* DirectAlphaShape2D.cpp:724-726: LBVH build, infinity points, neighbour count pass. */
void AlphaShape2D_init(AlphaShape2D* ashape);
/* DirectAlphaShape2D.cpp:729-732: neighbour fill, star Delaunay, alpha filter, compress. */
void AlphaShape2D_compute(AlphaShape2D* ashape);
/* DirectAlphaShape2D.cpp:735-737 */
uint32_t AlphaShape2D_get_nelem(const AlphaShape2D* ashape);
/* DirectAlphaShape2D.cpp:740-744: elems is nelem x 3 (Morton ids; a = owner, counter-clockwise). */
void AlphaShape2D_get_elem(const AlphaShape2D* ashape, uint32_t* elems);
/* DirectAlphaShape2D.cpp:746-753: nodes is nnodes x 2, Morton order. */
void AlphaShape2D_get_ordered_nodes(AlphaShape2D* ashape, float* nodes);
/* Additive: device points (x, y, unused, alpha) as nnodes float4. */
int AlphaShape2D_set_nodes_device(AlphaShape2D* ashape, uint32_t nnodes, const float* d_xy0a);
/* Additive: status bits of the last call (0 = ok). */
int AlphaShape2D_get_status(const AlphaShape2D* ashape);
/* Additive: out3 = {status bits, points whose neighbour fill stopped at the
 * reference's 250-id limit (DirectAlphaShape2D.cpp:351-354), exact in-circle calls}. */
int AlphaShape2D_get_counters(const AlphaShape2D* ashape, uint32_t* out3);
/* Additive (C++-only getPermutation, DirectAlphaShape2D.cpp:75-80). */
uint32_t AlphaShape2D_get_permutation(const AlphaShape2D* ashape, uint32_t* perm);
/* Additive (C++-only getEdge, DirectAlphaShape2D.cpp:90-98). */
uint32_t AlphaShape2D_get_nedge(const AlphaShape2D* ashape);
/* row nnodes+1, neig nedge, edge_is_bnd nedge (any may be NULL); returns nedge. */
uint32_t AlphaShape2D_get_edges(const AlphaShape2D* ashape, uint32_t* row, uint32_t* neig, uint8_t* edge_is_bnd);
/* Additive (C++-only getBoundaryNodes, DirectAlphaShape2D.cpp:101-105). */
uint32_t AlphaShape2D_get_boundary_nodes(const AlphaShape2D* ashape, uint8_t* is_bnd);
/* Additive diagnostics: nineig (star size incl. the 3 infinity ids), nkeep
 * (kept local triangles), neighbour rows (nnodes x width, UINT32_MAX padded). */
int AlphaShape2D_get_stars(const AlphaShape2D* ashape, uint32_t* nineig, uint8_t* nkeep, uint32_t* cand,
                           uint32_t width);
/* Additive: per-stage device milliseconds, ms6 = {LBVH, count pass, fill pass,
 * star, scans + size read-back, compress}, after set_profiling(1). */
int AlphaShape2D_set_profiling(AlphaShape2D* ashape, int on);
int AlphaShape2D_get_profile(AlphaShape2D* ashape, float* ms6);
/* Additive: caller-owned stream (NULL: the handle's own) and a wait on it. */
int AlphaShape2D_set_stream(AlphaShape2D* ashape, void* stream);
int AlphaShape2D_synchronize(AlphaShape2D* ashape);

/* ---------------------------------------------------------------- Mesh2D ---
 * Reference: src/mesh/mesh.cpp:806-862 (extern "C" block; the class is
 * include/mesh/mesh.hpp).  The Delaunay triangulation of the points and three
 * super nodes (the points' box centre -+ (largest extent + 10), mesh.cpp:
 * 92-105), each point's star verified against the whole point set; ids are
 * Morton ordered (Mesh2D_get_permutation), super nodes nnodes..nnodes+2. */
typedef struct Mesh2D Mesh2D;

/* mesh.cpp:806-809 */
Mesh2D* Mesh2D_create(void);
/* mesh.cpp:811-813 */
void Mesh2D_destroy(Mesh2D* mesh);
/* mesh.cpp:816-823: nodes is nnodes x 2 row-major (2 <= nnodes <= 16M, finite). */
void Mesh2D_set_nodes(Mesh2D* mesh, uint32_t nnodes, const float* nodes);
/* mesh.cpp:826-828: LBVH build, super nodes, every star = the super triangles. */
void Mesh2D_init(Mesh2D* mesh);
/* mesh.cpp:831-833: inserts the 8 Morton-order neighbours on each side. */
void Mesh2D_insert_morton_neighbors(Mesh2D* mesh);
/* mesh.cpp:837-839: one verification sweep (at most one point-LBVH query per
 * star triangle; a point found inside a circumcircle is inserted). */
void Mesh2D_insert_BVH_neighbors(Mesh2D* mesh);
/* mesh.cpp:841-843: later outputs leave out triangles with a super node. */
void Mesh2D_remove_super_nodes(Mesh2D* mesh);
/* mesh.cpp:845-847: verifies until every star triangle has an empty
 * circumcircle.  STREAM_ST_INCOMPLETE when a star stops unverified: out of
 * its 128 local ids (STREAM_ST_TET_CAP), or of its 512 queries or 65,536
 * LBVH node visits per sweep, or at a circle it cannot bound (coincident
 * points; such a query gives up after 8,192 points) (STREAM_ST_WALK_CAP). */
void Mesh2D_insert_iterative(Mesh2D* mesh);
/* mesh.cpp:849-852: compresses (each triangle once, by its smallest id). */
uint32_t Mesh2D_get_nelem(Mesh2D* mesh);
/* mesh.cpp:854-858: elems is nelem x 3 (owner first, counter-clockwise). */
void Mesh2D_get_elem(Mesh2D* mesh, uint32_t* elems);
/* mesh.cpp:860-862: nodes is nnodes x 2, Morton order. */
void Mesh2D_get_ordered_nodes(Mesh2D* mesh, float* nodes);
/* Additive: status bits of the calls since set_nodes. */
int Mesh2D_get_status(const Mesh2D* mesh);
/* Additive: out2 = {status bits, stars left unverified by the last sweep}. */
int Mesh2D_get_counters(const Mesh2D* mesh, uint32_t* out2);
/* Additive: ordered node i is input node perm[i]; returns nnodes. */
uint32_t Mesh2D_get_permutation(const Mesh2D* mesh, uint32_t* perm);
/* Additive: the three super nodes as x, y pairs. */
int Mesh2D_get_super_nodes(const Mesh2D* mesh, float* xy6);

/* ---------------------------------------------------------- Sphere3DLBVH ---
 * Reference: the C++ type Sphere3DLBVH (include/geometry/lbvh.hpp:50) and its
 * set_objects/build (lbvh.hpp:119-138,354-360); the reference has no C entry
 * points for it, so these are additive. */
typedef struct Sphere3DLBVH Sphere3DLBVH;
Sphere3DLBVH* Sphere3DLBVH_create(void);
void Sphere3DLBVH_destroy(Sphere3DLBVH* bvh);
/* xyzr: n x 4 host floats; bits 63 or 30; fit_point 1 = node boxes of centres. */
int Sphere3DLBVH_set_objects(Sphere3DLBVH* bvh, uint32_t n, const float* xyzr, int bits, int fit_point);
int Sphere3DLBVH_set_objects_device(Sphere3DLBVH* bvh, uint32_t n, const float* d_xyzr, int bits, int fit_point);
/* Enqueue the build (asynchronous on the handle's stream). */
int Sphere3DLBVH_build(Sphere3DLBVH* bvh);
/* Wait; *status receives the device status bits (may be NULL). */
int Sphere3DLBVH_synchronize(Sphere3DLBVH* bvh, uint32_t* status);
/* Additive: CUDA events between the build's stages (on = 1), and the last
 * profiled build's stage times in ms (box + Morton codes, radix sort, gather,
 * hierarchy + fit); returns the number of times written (<= cap). */
int Sphere3DLBVH_set_profiling(Sphere3DLBVH* bvh, int on);
uint32_t Sphere3DLBVH_get_profile(Sphere3DLBVH* bvh, float* ms, uint32_t cap);
/* Copy out (any pointer may be NULL): bb_glob[6], codes[n], perm[n], sep[n-1],
 * cil[n-1], leaf_parent[n], internal_parent[n-1], bboxes[(n-1) x 6], obj_m[n x 4]. */
int Sphere3DLBVH_get(Sphere3DLBVH* bvh, float* bb_glob, uint64_t* codes, uint32_t* perm, int32_t* sep,
                     uint8_t* cil, uint32_t* leaf_parent, uint32_t* internal_parent, float* bboxes, float* obj_m);

/* --------------------------------------------------------- Sphere3DTRBVH ---
 * Reference: the C++ type Sphere3DTRBVH (include/geometry/trbvh.hpp:55) and
 * its build (trbvh.hpp:299-679); additive C entry points.  Node ids: leaves
 * 0..n-1, internal nodes n..2n-2, root parent 2n. */
typedef struct Sphere3DTRBVH Sphere3DTRBVH;
Sphere3DTRBVH* Sphere3DTRBVH_create(void);
void Sphere3DTRBVH_destroy(Sphere3DTRBVH* t);
/* treelet_size in [3, 8] (reference 5); area3d 1 = xy+yz+zx, 0 = the reference's
 * ext_x*ext_y; rounds of restructuring (reference 3; 0 = Apetrei build only). */
int Sphere3DTRBVH_set_objects(Sphere3DTRBVH* t, uint32_t n, const float* xyzr, int treelet_size, int area3d,
                              int rounds);
int Sphere3DTRBVH_build(Sphere3DTRBVH* t);
int Sphere3DTRBVH_synchronize(Sphere3DTRBVH* t, uint32_t* status);
/* Additive: stage timing as for Sphere3DLBVH (box + Morton codes, radix sort,
 * gather, Apetrei build, treelet rounds). */
int Sphere3DTRBVH_set_profiling(Sphere3DTRBVH* t, int on);
uint32_t Sphere3DTRBVH_get_profile(Sphere3DTRBVH* t, float* ms, uint32_t cap);
int Sphere3DTRBVH_get(Sphere3DTRBVH* t, uint32_t* child_left, uint32_t* child_right, uint32_t* range_min,
                      uint32_t* range_max, uint32_t* parent, float* bboxes, uint32_t* subtree_size, float* sah,
                      uint32_t* root, float* obj_m);
/* Per object (Morton order): number of other spheres overlapping it. */
int Sphere3DTRBVH_count_overlaps(Sphere3DTRBVH* t, uint32_t* out);

/* ------------------------------------------------------------- numerics ---
 * Reference: include/numerics/csr.hpp:43-72, linear_system.hpp:41-58,
 * preconditioner.hpp:32-44, solver.hpp:46-65 (declarations) and the extern "C"
 * blocks of src/numerics/{csr,linear_system,preconditioner_jacobi,
 * conjugate_gradient}.cpp.  FP32 values and vectors, u32 indices. */
typedef struct DeviceCSR d_CSR;
typedef struct HostCSR h_CSR;
typedef struct LinearSystem LinSys;
typedef struct PrecJacobi PrecJacobi_st;
typedef struct ConjugateGradient SolverCG;

/* csr.cpp:105-107 */
d_CSR* d_csr_create(void);
/* csr.cpp:113-115 */
void d_csr_destroy(d_CSR* A);
/* csr.cpp:118-124: copies row[n+1], col[row[n]], val[row[n]]. */
h_CSR* h_csr_create(uint32_t n, const uint32_t* row, const uint32_t* col, const float* val);
/* csr.cpp:126-128 */
void h_csr_destroy(h_CSR* A);
/* csr.cpp:109-111 */
void d_csr_h2d(d_CSR* dcsr, const h_CSR* hcsr);
/* linear_system.cpp:27-32 */
LinSys* LinSys_create(void);
/* linear_system.cpp:34-36 */
void LinSys_destroy(LinSys* sys);
/* linear_system.cpp:38-43: shares A's device arrays (kept alive by reference
 * counting here), copies b (host, n floats). */
void LinSys_set(LinSys* sys, const d_CSR* A, const float* b);
/* preconditioner_jacobi.cpp:66-70 */
PrecJacobi_st* PrecJacobi_create(const d_CSR* A);
/* preconditioner_jacobi.cpp:72-74 */
void PrecJacobi_destroy(PrecJacobi_st* prec);
/* Additive (the reference leaves idiag uninitialised for a row without a
 * diagonal entry, preconditioner_jacobi.cpp:43-48): 0 when every row has a
 * nonzero diagonal entry with a finite inverse, else STREAM_ST_BAD_INPUT with
 * the number of rows that fail this in *bad_rows (may be NULL). */
int PrecJacobi_get_status(const PrecJacobi_st* prec, uint32_t* bad_rows);
/* conjugate_gradient.cpp:215-217 */
SolverCG* SolverCG_create(void);
/* conjugate_gradient.cpp:219-221 */
void SolverCG_destroy(SolverCG* solver);
/* conjugate_gradient.cpp:223-229: Jacobi-PCG (stop at sqrt(r.z) <= 1e-6, <= 10000
 * counted iterations); x host in/out; returns the reference's iteration counter. */
uint32_t SolverCG_jacobi_solve(SolverCG* solver, const LinSys* sys, const PrecJacobi_st* prec, float* x);
/* conjugate_gradient.cpp:231-237: unpreconditioned CG. */
uint32_t SolverCG_solve(SolverCG* solver, const LinSys* sys, float* x);
/* Additive: how the last solve ended: 1 the reference's stopping rule, 2 its
 * 10,000-iteration cap, 3 a non-finite r.z (breakdown), 0 no completed solve. */
int SolverCG_get_termination(const SolverCG* solver);

/* Additive: FP64 pressure systems (no reference counterpart; the reference has
 * no assembly and no FP64 solver). */
typedef struct PoissonSystem PoissonSystem;
PoissonSystem* PoissonSystem_create(void);
void PoissonSystem_destroy(PoissonSystem* ps);
/* P1 Laplacian on the computed alpha shape's tets (Morton ids), Dirichlet
 * (identity row, zero RHS, eliminated column) on its free-surface nodes.
 * rhs_kind 0: f = 1; 1: f = div u for u = sum_m a_m sin(k_m.x + phi_m), modes
 * nmodes x {kx, ky, kz, a.k, phi} (nmodes <= 8). */
int PoissonSystem_assemble(PoissonSystem* ps, const AlphaShape3D* mesh, int rhs_kind, const float* modes, int nmodes);
/* Host FP64 CSR + RHS. */
int PoissonSystem_set_csr(PoissonSystem* ps, uint32_t n, const uint32_t* row, const uint32_t* col,
                          const double* val, const double* b);
int PoissonSystem_get_size(const PoissonSystem* ps, uint32_t* n, uint32_t* nnz);
int PoissonSystem_get_csr(const PoissonSystem* ps, uint32_t* row, uint32_t* col, double* val, double* b);
/* method 0: FP64 Jacobi-PCG; 1: mixed-precision Jacobi-PCG; 2: mixed-precision
 * PCG with the learned FSAI preconditioner attached by PoissonSystem_set_fsai
 * (z = G^T G r), falling back to FP64 Jacobi-PCG when a segment fails to halve
 * the residual.  Methods 1 and 2 run FP32 iterations (FP32 SpMV and
 * preconditioner, FP64 dot products) in segments that each reduce the residual
 * by inner_rtol, or with inner_rtol <= 0 by max(1e-2, rtol ||b|| / (2 ||r||));
 * after each the correction is added to the FP64 x, the FP64 residual b - Ax
 * replaces the FP32 one and the iteration goes on with its search direction.
 * Stops at ||b - Ax|| <= rtol ||b||; "outer steps" counts the segments.  x
 * host FP64 in/out or NULL.
 * Method 3 is method 2's refinement with the Kolotilina-Yeremin FSAI on A's
 * lower pattern instead of the network's G: row i of G solves A[J,J] g = e_i
 * (J the columns j <= i of row i) scaled to diag(G A G^T) = 1 (no model).
 * report[6] = {iterations, outer steps, true relative residual, device ms
 * (methods 2 and 3: including the preconditioner's set-up and inference or
 * local solves when they ran), converged, fallback used}. */
int PoissonSystem_solve(PoissonSystem* ps, int method, double rtol, uint32_t maxit, double inner_rtol, double* x,
                        double* report);
int PoissonSystem_get_solution(const PoissonSystem* ps, double* x);
int PoissonSystem_assembly_stats(const PoissonSystem* ps, uint32_t* isolated);
/* Node coordinates (n x 3, FP64) for a system set with PoissonSystem_set_csr;
 * assembled systems take them from the mesh. */
int PoissonSystem_set_coords(PoissonSystem* ps, const double* xyz);

/* Additive: learned FSAI preconditioner (no reference counterpart; the
 * reference's preconditioner interface, include/numerics/preconditioner.hpp:48-72,
 * has Jacobi only).  A per-edge MLP 16 -> 64 -> 64 -> 64 -> 1 (tanh-form GELU,
 * bf16 tensor-core operands, fp32 accumulation) maps features of each lower
 * entry (i, j) of A (a_ij / sqrt(a_ii a_jj), log-diagonals, relative position
 * and distance over the mean edge length, boundary fractions, [i == j]) to
 * G_ij; M = G^T G.  Parameters: one float vector of FsaiModel_param_count()
 * values, W1[16][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] w4[64] b4. */
#define STREAM_FSAI_PARAM_COUNT 9473u
typedef struct FsaiModel FsaiModel;
uint32_t FsaiModel_param_count(void);
FsaiModel* FsaiModel_create(void); /* all-zero parameters: M = Jacobi */
void FsaiModel_destroy(FsaiModel* m);
int FsaiModel_set_params(FsaiModel* m, const float* params, uint32_t count);
int FsaiModel_get_params(const FsaiModel* m, float* params, uint32_t count);
int FsaiModel_reset_optimizer(FsaiModel* m);
/* Training loss of the model: STREAM_FSAI_LOSS_RESIDUAL (the default)
 * sum_p ||G A G^T z_p - z_p||^2 / (16 n), or STREAM_FSAI_LOSS_KAPORIN
 * log(t / n) - (2/n) sum_i log G_ii with t = sum_p z_p^T G A G^T z_p / 16 (the
 * log of Kaporin's condition number of G A G^T up to log(det A) / n, the
 * functional the Kolotilina-Yeremin FSAI minimises).  Unknown kinds: error. */
#define STREAM_FSAI_LOSS_RESIDUAL 0u
#define STREAM_FSAI_LOSS_KAPORIN 1u
int FsaiModel_set_loss(FsaiModel* m, uint32_t kind);
/* What the network's output corrects: STREAM_FSAI_BASE_NONE (the default;
 * G_ij = out / sqrt(a_jj), G_ii = exp(out) / sqrt(a_ii), zero output =
 * Jacobi) or STREAM_FSAI_BASE_KY, the Kolotilina-Yeremin G K of the system
 * (G_ij = K_ij + out / sqrt(a_jj), G_ii = exp(out) K_ii, zero output = K;
 * K_ij sqrt(a_jj) is input feature 10).  Unknown kinds: error. */
#define STREAM_FSAI_BASE_NONE 0u
#define STREAM_FSAI_BASE_KY 1u
int FsaiModel_set_base(FsaiModel* m, uint32_t base);
int FsaiModel_get_base(const FsaiModel* m, uint32_t* base);
/* The model's loss over 16 probes z_p (Rademacher from seed, or probes: host
 * n x 16 row-major when non-NULL) and its gradient (grad: host
 * float[param_count] or NULL). */
int FsaiModel_loss_grad(FsaiModel* m, PoissonSystem* ps, uint64_t seed, const float* probes, double* loss,
                        float* grad);
/* One Adam step (beta 0.9/0.999) on the loss of ps; clip > 0 clips the
 * gradient's global norm. */
int FsaiModel_train_step(FsaiModel* m, PoissonSystem* ps, uint64_t seed, float lr, float clip, double* loss);
/* One Adam step on the mean loss (and mean gradient) of count systems, the
 * probes of system i seeded with seed + i; *loss = the mean loss. */
int FsaiModel_train_batch(FsaiModel* m, PoissonSystem* const* systems, uint32_t count, uint64_t seed, float lr,
                          float clip, double* loss);
/* Attach (or with NULL detach) the model used by method 2; the model must stay
 * alive while attached.  The next method-2 solve builds the preconditioner
 * (set-up and inference, both inside its reported time); later solves reuse it
 * until the matrix or the model's parameters change. */
int PoissonSystem_set_fsai(PoissonSystem* ps, FsaiModel* m);
/* G aligned with the CSR (g[k] = G_ij for k = (i, j <= i), G_ji for j > i; nnz
 * floats; needs an attached model), the features of the lower entries
 * (n_lower x 16 floats) and their count; each pointer may be NULL. */
int PoissonSystem_get_fsai(PoissonSystem* ps, float* g, float* features, uint32_t* n_lower);
/* stats[4] = {set-up ms, inference ms, fallback used by the last solve, lower entries}. */
int PoissonSystem_fsai_stats(const PoissonSystem* ps, double* stats);
/* The Kolotilina-Yeremin G of method 3 (built if needed), aligned with the CSR
 * like PoissonSystem_get_fsai (g: nnz floats or NULL), and the number of rows
 * left diagonal (1/sqrt(a_ii)) because their lower pattern has more than 24
 * entries or their local block lost positivity in float (diag_rows or NULL). */
int PoissonSystem_get_ky(PoissonSystem* ps, float* g, uint32_t* diag_rows);

/* Additive: PFEM step loop (no reference counterpart; the reference meshes
 * given clouds).  Particles (FP64, particle order) are advected every step by
 * an analytic divergence-free Taylor-Green field
 *   u = amp R^T (sin kx' cos ky' cos kz', -cos kx' sin ky' cos kz', 0),
 *   x' = R (x - c),  tg = {R[9] row-major, c[3], k, amp}
 * (explicit Euler), remeshed (LBVH + alpha shape, free surface), and the P1
 * pressure system (Dirichlet on the free surface, RHS = div of the predictor
 * modes set by PfemLoop_set_rhs_modes) is assembled and solved to rtol with
 * the learned-FSAI mixed solver (Jacobi-PCG fallback) when a model is
 * attached, else with FP64 Jacobi-PCG.  Each solve starts from the previous
 * step's pressure at the same particles (zero on the free surface); the first
 * one after PfemLoop_set_particles starts from zero unless
 * PfemLoop_set_pressure gave one. */
typedef struct PfemLoop PfemLoop;
/* Euler steps of the field on host positions (n x 3 FP64, in place), on the GPU. */
int stream_b200_advect_taylor_green(uint32_t n, double* xyz, const double* tg, double dt, uint32_t steps);
PfemLoop* PfemLoop_create(void); /* default field: R = I, c = 0, k = 2 pi, amp = 0.5 */
void PfemLoop_destroy(PfemLoop* loop);
int PfemLoop_set_particles(PfemLoop* loop, uint32_t n, const double* xyz, float alpha);
int PfemLoop_get_particles(const PfemLoop* loop, double* xyz);
int PfemLoop_set_flow(PfemLoop* loop, const double* tg);
int PfemLoop_set_rhs_modes(PfemLoop* loop, const float* modes, int nmodes);
int PfemLoop_set_fsai(PfemLoop* loop, FsaiModel* m);
/* Fractional-step dynamics instead of the Taylor-Green advection (Chorin's
 * projection on the P1 mesh of the particles, one per step):
 *   u* = u + dt (g + nu lap u);  K p = -(rho/dt) D u*;  u = u* - (dt/rho) grad p;
 *   x += dt u,
 * lumped mass, explicit viscosity, p = 0 on the free surface away from the
 * box walls, zero normal velocity at the walls (nodes within alpha/2 of a
 * face), particles kept inside the box.  params[11] = {g[3], nu, rho,
 * lo[3], hi[3]}; NULL turns it off.  Velocities start at zero. */
int PfemLoop_set_physics(PfemLoop* loop, const double* params);
/* Particle velocities, n x 3 FP64, particle order. */
int PfemLoop_get_velocity(const PfemLoop* loop, double* uvw);
int PfemLoop_set_velocity(PfemLoop* loop, const double* uvw);
/* One step of dt.  report[12] = {advect ms (with dynamics: predictor,
 * correction and particle move), remesh ms, assembly ms, preconditioner ms,
 * solve ms, step ms, iterations, fallback used, nodes, tets, true relative
 * residual, converged}. */
int PfemLoop_step(PfemLoop* loop, double dt, double rtol, double* report);
/* Pressure of the last step in particle order. */
int PfemLoop_get_pressure(PfemLoop* loop, double* p);
/* Initial guess of the next solve, particle order (n values; e.g. the
 * pressure saved with a checkpoint). */
int PfemLoop_set_pressure(PfemLoop* loop, const double* p);
/* stats[2] = {steps done, steps that needed the fallback}. */
int PfemLoop_stats(const PfemLoop* loop, uint64_t* stats);
/* Borrowed handles of the current step's mesh and system (valid until the next step). */
AlphaShape3D* PfemLoop_mesh(PfemLoop* loop);
PoissonSystem* PfemLoop_system(PfemLoop* loop);

#ifdef __cplusplus
}
#endif
#endif /* STREAM_B200_H */
