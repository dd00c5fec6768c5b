/* lbm_b200.h -- C ABI of the B200 (sm_100a) D3Q19 TRT kernels.
 *
 * The drop-in boundary is the reference benchmark's own kernel-table API:
 *
 *   typedef struct KernelFunctions_ { char Name[128];
 *       void (*Init)(LatticeDesc *, KernelData **, Parameters *);
 *       void (*Deinit)(LatticeDesc *, KernelData **); } KernelFunctions;
 *                                                   (src/KernelFunctions.h:49-54)
 *
 * Each CUDA kernel below is one Init/Deinit pair with exactly those
 * signatures. Init builds the device layout from the LatticeDesc mask, uploads
 * it, and installs in the returned KernelData (src/Kernel.h:187-211):
 *   Kernel   runs cd->MaxIterations time steps on the GPU (the AA kernels, as
 *            in the reference, advance in even/odd pairs), synchronises, sets
 *            Duration, and leaves a host mirror valid for GetNode;
 *   GetNode / SetNode, BoundaryConditionsGetPdf / SetPdf
 *            read and write the logical PDFs of a node through the mirror
 *            (SetNode marks it for upload before the next Kernel call);
 *   LoopBalance  the kernel's algorithmic bytes per fluid-lattice update.
 * Errors print a message and exit(1), as the reference does.
 *
 * The structs are layout-compatible with the reference's (PdfT = double). If
 * the reference's Kernel.h has been included first, its definitions are used.
 *
 * Library: liblbmb200.so (lbm-benchmark-kernels_b200/), built for sm_100a.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef __KERNEL_H__
/* ---- reference-compatible types (src/Lattice.h:33-55, src/Kernel.h:172-222) ---- */
typedef double PdfT;
typedef int LatticeT;

enum { LAT_CELL_OBSTACLE = 0, LAT_CELL_FLUID = 1, LAT_CELL_INLET = 2, LAT_CELL_OUTLET = 4 };

typedef struct LatticeDesc_ {
	int Dims[3];
	LatticeT *Lattice;
	int nCells;
	int nFluid;
	int nObst;
	int nInlet;
	int nOutlet;
	int PeriodicX;
	int PeriodicY;
	int PeriodicZ;
	const char *Name;
} LatticeDesc;

typedef struct CaseData_ {
	PdfT Omega;
	PdfT RhoIn;
	PdfT RhoOut;
	PdfT Ux;
	PdfT Uy;
	PdfT Uz;
	PdfT XForce;
	int MaxIterations;
	int VtkOutput;
	int VtkModulus;
	int StatisticsModulus;
} CaseData;

typedef struct KernelData_ {
	PdfT *Pdfs[2];
	PdfT *SrcPdfs;
	PdfT *DstPdfs;
	PdfT *PdfsActive;
	int Dims[3];
	int GlobalDims[3];
	int Offsets[3];
	int *ObstIndices;
	int nObstIndices;
	int *BounceBackPdfsSrc;
	int *BounceBackPdfsDst;
	int nBounceBackPdfs;
	double LoopBalance;
	double Duration;
	void (*BoundaryConditionsGetPdf)(struct KernelData_ *kd, int x, int y, int z, int dir, PdfT *pdf);
	void (*BoundaryConditionsSetPdf)(struct KernelData_ *kd, int x, int y, int z, int dir, PdfT pdf);
	void (*GetNode)(struct KernelData_ *kd, int x, int y, int z, PdfT *pdfs);
	void (*SetNode)(struct KernelData_ *kd, int x, int y, int z, PdfT *pdfs);
	void (*Kernel)(LatticeDesc *ld, struct KernelData_ *kd, CaseData *cd);
} KernelData;

typedef struct Parameters_ {
	int nArgs;
	char **Args;
	int nKernelArgs;
	char **KernelArgs;
} Parameters;
#endif /* __KERNEL_H__ */

/* ---- kernel-table rows (drop-ins for src/KernelFunctions.h:56-188) ----
 * Kernel arguments (after "--" on the command line, Parameters.KernelArgs):
 *   -lambda <v|a/b>   TRT magic parameter (default 1/12, the value the
 *                     reference hard-codes, e.g. src/BenchKernelD3Q19Aa.c:71)
 *   -blk <n>, -blk-x/-blk-y/-blk-z <n>
 *                     list kernels: blocked numbering of the fluid nodes, as
 *                     src/BenchKernelD3Q19ListAaPvCommon.c:631-656
 *   -pad auto|no|m+o[,m+o]*  list kernels: SoA padding (src/Padding.c:19-193)
 *   -bs <n>           threads per block of the list kernels (default 256)
 */

/* "cuda-aa-soa": AA pattern, full array, SoA. Replaces D3Q19AaInit_AaSoA /
 * D3Q19AaDeinit_AaSoA (src/BenchKernelD3Q19Aa.h:33-37, registered as "aa-soa"
 * at src/KernelFunctions.h:171-175). */
void D3Q19CudaAaInit_AaSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaAaDeinit_AaSoA(LatticeDesc *ld, KernelData **kernelData);

/* "cuda-list-aa-pv-soa": AA pattern over the fluid-node list with a push
 * adjacency. Replaces D3Q19ListAaPvInit_PushSoA / ..Deinit_PushSoA
 * (src/BenchKernelD3Q19ListAaPv.h, registered at src/KernelFunctions.h:58-62). */
void D3Q19CudaListAaPvInit_PushSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListAaPvDeinit_PushSoA(LatticeDesc *ld, KernelData **kernelData);

/* "cuda-list-pull-split-nt-1s-soa" / "-2s-soa": two-grid pull over the
 * fluid-node list. Replace D3Q19ListPullSplitNt1SInit_PullSoA,
 * D3Q19ListPullSplitNt2SInit_PullSoA and D3Q19ListPullSplitNtDeinit_PullSoA
 * (src/BenchKernelD3Q19ListPullSplitNt.h, src/KernelFunctions.h:96-105). On the
 * GPU both names run the same one-thread-per-node kernel. */
void D3Q19CudaListPullSplitNt1SInit_PullSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListPullSplitNt2SInit_PullSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListPullSplitNtDeinit_PullSoA(LatticeDesc *ld, KernelData **kernelData);

/* "cuda-list-aa-soa" / "cuda-list-aa-ria-soa": the reference's other list-AA
 * rows (src/KernelFunctions.h:63-72: D3Q19ListAaInit_PushSoA,
 * D3Q19ListAaRiaInit_PushSoA and their Deinit). Same layout and arithmetic as
 * list-aa-pv-soa; on the GPU they run the list AA kernels. */
void D3Q19CudaListAaInit_PushSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListAaDeinit_PushSoA(LatticeDesc *ld, KernelData **kernelData);
void D3Q19CudaListAaRiaInit_PushSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListAaRiaDeinit_PushSoA(LatticeDesc *ld, KernelData **kernelData);

/* "cuda-list-push-soa" / "cuda-list-pull-soa": two-grid list kernels, push or
 * pull adjacency, SoA padding without the pull-split cache-line pad. Replace
 * D3Q19ListInit_PushSoA / D3Q19ListInit_PullSoA and their Deinit
 * (src/BenchKernelD3Q19List.c, registered at src/KernelFunctions.h:106-120). */
void D3Q19CudaListInit_PushSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListDeinit_PushSoA(LatticeDesc *ld, KernelData **kernelData);
void D3Q19CudaListInit_PullSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaListDeinit_PullSoA(LatticeDesc *ld, KernelData **kernelData);

/* "cuda-push-soa" / "cuda-pull-soa": the two-grid full-array kernels
 * (src/BenchKernelD3Q19.c, registered at src/KernelFunctions.h:126-145 as
 * D3Q19Init_PushSoA / D3Q19Init_PullSoA and their Deinit), on the
 * full-array layout of cuda-aa-soa with a second grid; the reference's
 * bounce-back/periodic fix-up lists and body-force pass are folded into the
 * stores. GetNode of pull-soa views node x's PDF d at x - c_d, as the
 * reference's. */
void D3Q19CudaInit_PushSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaDeinit_PushSoA(LatticeDesc *ld, KernelData **kernelData);
void D3Q19CudaInit_PullSoA(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
void D3Q19CudaDeinit_PullSoA(LatticeDesc *ld, KernelData **kernelData);

/* The rows above as a table: {Name, Init, Deinit}, in the layout of the
 * reference's KernelFunctions (src/KernelFunctions.h:49-54). */
typedef struct LbmB200KernelFunctions_ {
	char Name[128];
	void (*Init)(LatticeDesc *ld, KernelData **kernelData, Parameters *params);
	void (*Deinit)(LatticeDesc *ld, KernelData **kernelData);
} LbmB200KernelFunctions;

const LbmB200KernelFunctions *lbm_b200_kernels(int *count);

/* ---- host helpers on the same path (src/Kernel.c, src/Geometry.c) ---- */

/* GeoCreateByStr (src/Geometry.c:37-88): box, channel, pipe, blocks[-n],
 * fluid, and (new) spheres[:seed:porosity:rmin:rmax], see lbm_geo_spheres. Allocates ld->Lattice (free with free()). Periodic flags are recorded
 * in ld before the geometry forces its own, as in the reference. Returns 0, or
 * -1 with a message for an unknown geometry or a bad block size. */
int lbm_geo_create(const char *geometryType, int dims[3], int periodic[3], LatticeDesc *ld);

/* KernelSetInitialDensity / KernelSetInitialVelocity (src/Kernel.c:258-438). */
void lbm_set_initial_density(LatticeDesc *ld, KernelData *kd, CaseData *cd);
void lbm_set_initial_velocity(LatticeDesc *ld, KernelData *kd, CaseData *cd);

/* KernelVerifiy (src/Kernel.c:511-625): L2 norm of the relative error of the
 * x-velocity profile at x = nX/2 against plane Poiseuille flow. Writes
 * flow-profile.dat into the current directory when write_file is set. */
double lbm_verify(LatticeDesc *ld, KernelData *kd, CaseData *cd, int write_file);

/* KernelDensity (src/Kernel.c:209-254): mean density over the fluid nodes. */
double lbm_density(KernelData *kd, LatticeDesc *ld);

/* VtkWrite (src/Vtk.c:51-245): legacy VTK file of the current state through
 * GetNode -- cell flags, density, velocity (with the F/2 shift of the
 * reference's VERIFICATION builds) -- byte for byte the reference's format.
 * lbm_vtk_write writes vtk/file-%04d.vtk (creating vtk/), as the reference;
 * lbm_vtk_write_file writes `path`. Return 0 or -1. The CUDA rows' Kernel
 * writes these files itself when cd->VtkOutput is set: before the first step
 * (label -1), after each step pair (AA forms) or step (pull) whose first step
 * index is a multiple of cd->VtkModulus (label: that index), and after the
 * last step (label MaxIterations). */
int lbm_vtk_write(LatticeDesc *ld, KernelData *kd, CaseData *cd, int iteration);
int lbm_vtk_write_file(LatticeDesc *ld, KernelData *kd, CaseData *cd, int iteration, const char *path);

/* ---- B200 additions with no counterpart in the reference ---- */

/* Seeded packing of solid spheres in a fully periodic box: random sequential
 * addition of non-overlapping spheres (radii uniform in [rmin, rmax]) until
 * the voxel porosity reaches `porosity`, or until `rsaAttempts` placements in
 * a row have failed (jammed); then spheres are added without the overlap test
 * until the target is met. Random numbers: splitmix64-seeded PCG32.
 * stats (optional, 4 doubles): achieved porosity, spheres placed without
 * overlap, spheres placed with overlap allowed, porosity at jamming (-1 if
 * the target was reached first). ld gets a malloc'ed mask (free with free())
 * and periodic flags 1,1,1. Returns 0, or -1 for bad arguments. */
int lbm_geo_spheres(const int dims[3], uint64_t seed, double porosity, double rmin, double rmax,
                    int rsaAttempts, LatticeDesc *ld, double *stats);

/* Device time (ms, CUDA events on the kernel's stream) of the time-step loop
 * of the last Kernel call; Duration holds the host wall time around the same
 * loop including the final synchronisation. */
double lbm_b200_last_device_ms(KernelData *kd);

/* Number of kernel launches of the last Kernel call. */
long lbm_b200_last_launches(KernelData *kd);

/* Bytes moved host->device and device->host by the last Kernel call (mirror
 * upload of a dirty mirror, download after the steps). List layouts move only
 * the node range [0, nFluid) of each direction's plane of nCells elements
 * (the padding behind the nodes holds no state): 19 * nFluid * element bytes
 * each way; full-array layouts move the whole array. */
void lbm_b200_last_copy_bytes(KernelData *kd, size_t *h2d, size_t *d2h);

/* Lost device state. The kernels' bounded waits (bulk copies into shared
 * memory) give up after a fixed number of polls and set a device error word
 * instead of hanging; a skipped tile sets it too. The calls below that read
 * the word (sync_mirror, time_steps, instance_moments, checkpoint_save, and
 * Kernel, which exits) then mark the instance's device state as lost: a copy
 * that arrived late may have landed in another block's shared memory, so
 * none of that launch's results can be trusted. While the state is lost,
 * every step entry point refuses with -4 (Kernel exits with a message),
 * sync_mirror keeps the mirror at the last good state and returns -4, and
 * checkpoint_save writes nothing (-4). Uploading a host state (set_field,
 * SetNode edits followed by a step call, or checkpoint_load) clears it. */

/* The -verify check of KernelVerifiy (src/Kernel.c:456-625) on the device:
 * the x-velocity slice at x = nX/2 and the Poiseuille L2 relative error,
 * summed over z with warp shuffles, from the instance's device PDFs (after
 * its pending steps; a dirty mirror is uploaded first). Moves only the nY x
 * nZ slice and the error to the host -- not the field, as a GetNode-based
 * check after a device-only run would. *err = the error norm; with
 * write_file also the reference's flow-profile.dat. Returns 0, -1 for a
 * lattice of other dimensions, -4 on a lost device state, or a CUDA error
 * code. */
int lbm_b200_verify_device(LatticeDesc *ld, KernelData *kd, CaseData *cd, int write_file, double *err);

/* Test hook for the rule above: writes `word` into the instance's device
 * error word from the host (after its pending work), as a bounded wait that
 * gave up would have; no kernel runs and nothing faults. Returns 0 or a CUDA
 * error code. */
int lbm_b200_inject_device_error(KernelData *kd, int word);

/* Runs n time steps without touching the host mirror (no upload, no download,
 * no synchronisation), for callers that keep the state on the device. Returns
 * 0, -4 on a lost device state, or a CUDA error code. */
int lbm_b200_step_device(KernelData *kd, CaseData *cd, int n);

/* Copies the device state into the host mirror (blocking); -4 (mirror
 * unchanged) on a lost device state. */
int lbm_b200_sync_mirror(KernelData *kd);

/* Marks the host mirror as changed, so the next Kernel call uploads it. */
void lbm_b200_mark_mirror_dirty(KernelData *kd);

/* Runs n time steps on the device and times them with CUDA events on the
 * instance's stream: *total_ms for the whole sequence, per_launch_ms[k]
 * (optional, n entries) for launch k. No mirror traffic. Returns 0, -1 when
 * the device error word is set after the steps, -4 on a lost device state,
 * or a CUDA error code. */
int lbm_b200_time_steps(KernelData *kd, CaseData *cd, int n, double *total_ms, double *per_launch_ms);

/* Number of kernel launches that n time steps take on this instance (the
 * size of lbm_b200_time_steps' per_launch_ms): AA kernels run whole even/odd
 * pairs of 2-4 launches (even step; odd step interior blocks without and with
 * reversed links; face shell), list AA 2 per pair, pull 1 per step. */
long lbm_b200_launches_for(KernelData *kd, int n);

/* Adjacency bytes one adjacency-driven launch of a list instance reads (the
 * list AA odd step, the push and the pull steps): the run-compressed
 * records -- one 18-entry row per run of consecutive nodes whose links all
 * advance by one (the reference's consecutive nodes, cut at 256-node tiles)
 * plus a 48-byte header per tile. 0 for the full-array kernels. */
long long lbm_b200_adjacency_bytes(KernelData *kd);

/* Copies a list instance's run-compressed adjacency to host memory:
 * tileOffsets (nTiles + 1 entries, 16-byte units; nTiles = ceil(nodes/256))
 * and records (lbm_b200_adjacency_bytes bytes). Either may be NULL. Per
 * tile: 8 words of run-head mask (bit k of word w: node 32 w + k of the tile
 * starts a run), 2 words holding the heads before each mask word (byte w),
 * 2 zero words, then one 18-entry row per head (even count); node n's link d
 * is its head's entry d plus n - head. Returns 0, -1 for the full-array
 * kernels, or a CUDA error code. */
int lbm_b200_run_records(KernelData *kd, uint32_t *tileOffsets, uint32_t *records);

/* ---- x-slabs of an AA-pattern lattice (one lattice over several GPUs) ----
 * No counterpart in the reference, whose kernels address one array; the
 * slabs reproduce the undivided lattice's run bit for bit.
 *
 * lbm_aa_slab_init: an AA instance (the cuda-aa-soa kernels, Parameters as
 * its Init) over the x range [x0, x1) of `global`, in local coordinates
 * (local x = x - x0; GetNode/SetNode/get_field use a LatticeDesc of the slab).
 * Link words come from the whole lattice, so a link into a neighbouring slab
 * is direct exactly when the global neighbour is fluid. haloLo / haloHi: the
 * x = x0 / x = x1-1 face borders a neighbour slab (on the lattice's own x
 * boundary only with a periodic axis: the ring's wrap). Returns NULL on
 * errors (lbm_b200_last_error).
 *
 * lbm_aa_list_slab_init: the same for the list AA kernel
 * (cuda-list-aa-pv-soa, any -precision): the slab's fluid cells are the
 * owned nodes (the kernel's blocked numbering over the slab), followed by
 * ghost nodes for the fluid cells of the neighbouring slabs that owned links
 * reach; adjacency follows the whole lattice's link rule.
 *
 * A step pair is: lbm_aa_slab_step(half 0, even step) on every slab; for
 * every halo face, lbm_aa_halo_pack(side, 0) -> send to the neighbour ->
 * lbm_aa_halo_unpack(side, 0) there; lbm_aa_slab_step(half 1, odd step); the
 * same exchange with phase 1. side 0 is the x0 face, 1 the x1-1 face.
 * Pack of (side 1, phase p) pairs with unpack of (side 0, phase p) on the
 * right-hand neighbour and vice versa. Messages are PDF elements in device
 * memory, in the slab's storage format moved bit for bit
 * (lbm_aa_halo_elem_bytes: 8 for FP64, 4 or 2 for the FP32 / FP16 list
 * storage): lbm_aa_halo_message(side, phase, send) of them go out (send = 1)
 * or come in (send = 0) through a face -- 5 x nY x nZ for full-array slabs,
 * the face's link count for list slabs (-1: no halo on that face);
 * lbm_aa_halo_count is the largest message of the slab. The functions
 * enqueue on `stream` (NULL: the instance's stream) and return 0 or an error
 * code; after steps on another stream, synchronise it before
 * lbm_b200_sync_mirror. */
KernelData *lbm_aa_slab_init(LatticeDesc *global, int x0, int x1, int haloLo, int haloHi, Parameters *params);
KernelData *lbm_aa_list_slab_init(LatticeDesc *global, int x0, int x1, int haloLo, int haloHi, Parameters *params);
void lbm_aa_slab_deinit(KernelData *kd);
long long lbm_aa_halo_count(KernelData *kd);
long long lbm_aa_halo_message(KernelData *kd, int side, int phase, int send);
int lbm_aa_halo_elem_bytes(KernelData *kd);
int lbm_aa_halo_pack(KernelData *kd, int side, int phase, void *buf, void *stream);
int lbm_aa_halo_unpack(KernelData *kd, int side, int phase, const void *buf, void *stream);
int lbm_aa_slab_step(KernelData *kd, CaseData *cd, int half, void *stream);

/* The odd step of a slab (lbm_aa_slab_step half 1) in two parts, so that the
 * phase-0 messages can travel while part 0 runs: part 0 updates the cells
 * whose odd step touches no halo slot (full-array slabs: the interior blocks;
 * list slabs: the inner tile range, see lbm_aa_list_slab_layout) and needs no
 * message; part 1 updates the rest and must follow the phase-0 unpack. Call
 * each part once per pair; the phase-1 pack follows part 1. Together they
 * equal lbm_aa_slab_step(half 1). Returns 0 or an error code. */
int lbm_aa_slab_odd_part(KernelData *kd, CaseData *cd, int part, void *stream);

/* The even step (half 0) in the same two parts, so that the phase-1
 * messages of the previous pair can travel while part 0 runs: part 0 updates
 * the cells whose slots no halo message touches (full-array slabs: x in
 * [1, nX-2]; list slabs: the inner tile range; with FP16 storage both parts
 * use the per-node even kernel instead of the staged one); part 1 the rest,
 * after the phase-1 unpack and before the phase-0 pack. Returns 0 or an
 * error code. */
int lbm_aa_slab_even_part(KernelData *kd, CaseData *cd, int part, void *stream);

/* The layout lbm_aa_list_slab_init builds, on the host only (no CUDA call):
 * counts[0..8] = owned nodes, ghost nodes, nCells, then the lengths of the
 * own / ghost slot lists of side 0 and of side 1 (-1: no halo), then the
 * inner tile range [counts[7], counts[8]) of 256-node tiles whose nodes link
 * to no ghost node (lbm_aa_slab_odd_part's part 0; empty when the face
 * tiles are not all at the two ends of the numbering). Non-NULL
 * arrays receive the slab's numbering (x1-x0 by nY by nZ cells, x fastest;
 * obstacles 0xffffffff), the adjacency (owned nodes x 18, indices into
 * f[d * nCells + node]) and the four slot lists: own = the owned slots the
 * neighbour's face cells reach through that face (sent in phase 0, received
 * in phase 1), ghost = the ghost slots this slab's face cells reach
 * (received in phase 0, sent in phase 1). Returns 0 or a negative error. */
int lbm_aa_list_slab_layout(const LatticeDesc *global, int x0, int x1, int haloLo, int haloHi, Parameters *params,
                            long long *counts, uint32_t *grid, uint32_t *adj, uint32_t *ownLo, uint32_t *ghostLo,
                            uint32_t *ownHi, uint32_t *ghostHi);

/* Runs a kernel that waits, with a bound of `polls` reads, on a device flag
 * that nothing sets: the wait runs out, the kernel records error bit 2 in its
 * error word and returns, and *status receives the word (2). The same bounded
 * pattern guards every device wait of the library (the adjacency bulk copies),
 * whose error word the host checks after each Kernel call. Returns 0 or a
 * CUDA error code. */
int lbm_b200_selftest_bounded_wait(unsigned polls, int *status);

/* Selects the CUDA device used by subsequent Init calls of this thread. */
int lbm_b200_set_device(int device);

/* Device state of a list-kernel instance: the current PDF array (list
 * layout, f[d * nCells + n]), its padded cell count and node count, and the
 * instance's CUDA stream. Returns -1 for the full-array kernel. */
int lbm_b200_device_state(KernelData *kd, double **pdfs, long long *nCells, int *nFluid, void **stream);

/* FP64 conservation sums over the fluid nodes of a list-layout PDF array on
 * the device: out_device[0..3] = {sum rho, sum j_x, sum j_y, sum j_z}, with
 * rho = sum_i f_i and j = sum_i c_i f_i per node (the sums KernelDensity and
 * KernelStatisticsAdv form through GetNode, src/Kernel.c:209-254,633-755).
 * Fixed reduction tree: the result depends only on the field. Allocates a
 * scratch of 4 doubles per 256 nodes with cudaMalloc; stream may be NULL.
 * Synchronises the stream. Returns 0, or a CUDA error code / -1. */
int lbm_b200_moments_device(const double *pdfs, long long nCells, int nFluid, double *out_device, void *stream);

/* The same sums for a list-kernel instance, into host memory (out[0..3]);
 * waits for the instance's pending steps. With FP32/FP16 storage the stored
 * deviations from the weights are summed in FP64 and the node count added to
 * the mass. Returns 0, -1 for the full-array kernels, -4 on a lost device
 * state, or a CUDA error code. */
int lbm_b200_instance_moments(KernelData *kd, double *out);

/* Checkpoint / restart of an instance (no counterpart in the reference):
 * _save writes the current state -- a header (kernel, storage, lattice
 * dimensions and periodicity, a hash of the lattice mask, step parity,
 * Lambda; host byte order) and the PDF array exactly as the device holds it,
 * with an FNV-1a checksum; pending SetNode edits are part of the state. _load
 * restores it into an instance of the same kernel, storage, lattice
 * (geometry, not only its counts) and Lambda, so that the run continues bit
 * for bit. Return 0; -1 I/O error; -2 the file does not match the instance;
 * -3 checksum mismatch (state unchanged); -4 (_save) on a lost device state;
 * or a CUDA error code. */
int lbm_b200_checkpoint_save(KernelData *kd, const char *path);
int lbm_b200_checkpoint_load(KernelData *kd, const char *path);

/* Last CUDA error string seen by the library ("" if none). */
const char *lbm_b200_last_error(void);

/* Logical PDFs of every fluid cell through GetNode / SetNode: 19 doubles per
 * lattice cell, cells x fastest (src/Lattice.h:60-76), obstacle cells skipped. */
void lbm_b200_get_field(KernelData *kd, LatticeDesc *ld, double *out);
void lbm_b200_set_field(KernelData *kd, LatticeDesc *ld, const double *in);

/* Host-built list layout of a list-kernel instance: fluid-node numbering
 * (nX*nY*nZ entries, obstacles 0xffffffff), adjacency (nFluid*18, the
 * reference's order and index encoding), node and padded cell counts.
 * Returns -1 for the full-array kernel. */
int lbm_b200_list_layout(KernelData *kd, const uint32_t **grid, const uint32_t **adj, int *nFluid, int *nCells);

/* The same sums for callers that cannot allocate device memory: code that
 * runs while another component owns the device allocator, or that may only
 * use the buffers its host application hands it. Has no counterpart in the
 * reference. The reduction's scratch is a fixed 2 MiB array inside the
 * library (held by every GPU that loads it until the process exits), so a call
 * accepts at most 16,777,216 fluid nodes and returns -2 (with a message) above
 * that. Allocates nothing; does not synchronise (the result is ready when the
 * stream is). The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture; the
 * address is cached for the process, which assumes the device's context is
 * not reset (cudaDeviceReset) meanwhile. Calls share the array: calls that
 * overlap on the GPU race. A CUDA error already pending from earlier work is
 * returned without enqueueing anything. Returns 0, -1 for bad arguments, or a
 * CUDA error code. */
int lbm_b200_moments_noalloc(const double *pdfs, long long nCells, int nFluid, double *out_device, void *stream);

/* Host layout builders (no GPU needed), exported for the parity tests:
 * SoA padding (src/Padding.c:195-244), list numbering + adjacency
 * (src/BenchKernelD3Q19ListAaPvCommon.c:587-792; pull variant
 * src/BenchKernelD3Q19ListPullSplitNtCommon.c:548-755). */
int lbmh_pad_cells(int nCells, int pdfBytes, const char *padStr);
int lbmh_list_build(const LatticeDesc *ld, int pull, const int blk[3], int nCells,
                    uint32_t *grid, uint32_t *coords, uint32_t *adj);

/* The same layout built on the GPU (what the list rows' Init and
 * lbm_batch_add use): numbering in the blocked order by a prefix sum over the
 * cells, then each node's 18 links; host mask in, host grid (nX*nY*nZ) and
 * adjacency (ld->nFluid*18) out, bit-identical to lbmh_list_build. Returns
 * the fluid node count, -1 on a CUDA error, -2 when the mask holds more
 * non-obstacle cells than ld->nFluid (nothing written to adj). */
int lbm_b200_list_build(const LatticeDesc *ld, int pull, const int blk[3], int nCells, uint32_t *grid,
                        uint32_t *adj);

/* ---- Batched domains (no counterpart in the reference) ----
 * Many independent porous domains of uneven size, each with its own list
 * layout (push adjacency as the list AA kernel, node range padded to tiles of
 * 256 nodes) in its own device allocations, advanced together by one even and
 * one odd launch per step pair over a device table of tile records (a
 * persistent grid, or one block per tile). Storage fp32 (1) or fp16
 * deviations (2), FP32 arithmetic. The kernels read the table and its length
 * from device memory, so CUDA graphs captured for a step count stay valid as
 * domains are admitted and retired (until the table outgrows its allocation
 * or the one-block-per-tile grid, when they are captured again). */
void *lbm_batch_create(int storage, double budgetGB, int maxDomains);
void lbm_batch_destroy(void *batch);
/* Admits a domain at rest (f = w); returns its slot, -1 if the HBM budget is
 * exhausted, -2 if every slot is taken, other negatives on errors. */
int lbm_batch_add(void *batch, const LatticeDesc *ld, double omega, double lambda, double xforce);
int lbm_batch_remove(void *batch, int slot);
int lbm_batch_reset(void *batch, int slot);
/* Enqueues nsteps (rounded up to even) steps of every active domain; with
 * use_graph the sequence is replayed from a captured CUDA graph. */
int lbm_batch_step(void *batch, int nsteps, int use_graph);
int lbm_batch_sync(void *batch);
/* FP64 {rho, jx, jy, jz} sums of every slot: out has maxDomains * 4 doubles. */
int lbm_batch_moments(void *batch, double *out);
int lbm_batch_get_field(void *batch, int slot, double *out);
int lbm_batch_set_field(void *batch, int slot, const double *in);
/* which: 0 even, 1 odd, 2 both; threads 64/128/256 (nodes per thread =
 * 256 / threads); blocks = persistent grid size, 0 = one block per tile. */
int lbm_batch_set_launch(void *batch, int which, int threads, int blocks);
void lbm_batch_get_launch(void *batch, int *out6);
int lbm_batch_time_steps(void *batch, int nsteps, double *ms);
/* Autotuner over block size x nodes per thread x grid (2..6 persistent
 * blocks per SM, or 0 = one block per tile); rows of {which, threads,
 * nodesPerThread, blocks, ms}; keeps the fastest. */
int lbm_batch_tune(void *batch, int trialSteps, double *results, int maxRows);
/* Checkpoint / restart of one resident domain: its PDFs in the batch's
 * storage format plus its lattice size and relaxation parameters. _load
 * needs an active slot admitted from the same lattice with the same omega,
 * Lambda and force. Return codes as lbm_b200_checkpoint_save / _load. */
int lbm_batch_checkpoint_save(void *batch, int slot, const char *path);
int lbm_batch_checkpoint_load(void *batch, int slot, const char *path);
size_t lbm_batch_bytes_used(void *batch);
long long lbm_batch_launches(void *batch);
int lbm_batch_active_domains(void *batch);
int lbm_batch_fluid_nodes(void *batch, int slot);
const char *lbm_batch_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
