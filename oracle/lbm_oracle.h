/* lbm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's D3Q19 TRT update (lattice Boltzmann
 * benchmark kernels, src/): geometry masks, the AA full-array kernel with its
 * ghost layer and fix-up lists, the list numbering / padding / adjacency, the
 * list AA and list pull kernels, the body force, the -verify initialisation and
 * the Poiseuille check. Plain C99, no FP contraction, left-to-right sums in the
 * reference's scalar order, so FP64 results are bit-identical to the
 * reference's scalar kernels.
 *
 * Pinned against the reference itself (compiled from its sources by
 * oracle/Makefile into oracle/_ref/) by tests/test_oracle_pin.py, and against
 * the committed fixtures in tests/golden/.
 *
 * Only tests/, bench.py's cpu_baseline leg and __graft_entry__.smoke() may load
 * this library, and only as a checker.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* geometry types, numbered as the reference's GEO_TYPES (src/Geometry.h:33-42) */
enum { ORC_GEO_BOX = 0, ORC_GEO_CHANNEL = 1, ORC_GEO_PIPE = 2, ORC_GEO_BLOCKS = 3, ORC_GEO_FLUID = 4 };

/* kernels restated */
/* LIST_PULL is the pull-split layout (padding plus the cache-line pad of
 * src/BenchKernelD3Q19ListPullSplitNtCommon.c:494-496); LIST_PUSH2 and
 * LIST_PULL2 are the two-grid list kernels list-push-soa / list-pull-soa
 * (src/BenchKernelD3Q19List.c, layout src/BenchKernelD3Q19ListCommon.c:330-600,
 * padding only). */
/* PUSH_FA / PULL_FA: the two-grid full-array kernels push-soa / pull-soa
 * (src/BenchKernelD3Q19.c, layout and fix-up lists
 * src/BenchKernelD3Q19Common.c:291-670). */
enum { ORC_KERNEL_AA = 0, ORC_KERNEL_LIST_AA = 1, ORC_KERNEL_LIST_PULL = 2, ORC_KERNEL_LIST_PUSH2 = 3,
       ORC_KERNEL_LIST_PULL2 = 4, ORC_KERNEL_PUSH_FA = 5, ORC_KERNEL_PULL_FA = 6 };

/* init modes */
enum { ORC_INIT_ZERO = 0, ORC_INIT_VERIFY = 1, ORC_INIT_PDFS = 2 };

/* mask + counts. info_out: nFluid, nObst, nInlet, nOutlet, ldPeriodic x/y/z,
 * bits of the periodic flags written back to the caller (x=1,y=2,z=4). */
int orc_geometry(int type, int block_size, const int dims[3], const int periodic[3],
                 int *lattice_out, int *info_out);

/* nCells after the reference's SoA padding. pad_mode: 0 auto, 1 none,
 * 2 explicit pairs (n_pairs modulus/offset pairs in bytes). */
int orc_pad_cells(int n_cells, int pdf_bytes, int pad_mode, int n_pairs, const int *modulus, const int *offset);

/* List numbering and adjacency for the push (list AA) or pull (pull-split)
 * propagation model. grid_out: nX*nY*nZ (obstacles 0xffffffff), adj_out:
 * nFluid*18, counts_out: nFluid, nCells. blk: blocking (0 = none). */
int orc_list_layout(int pull, const int dims[3], const int periodic[3], const int *lattice,
                    const int blk[3], int pad_mode, int n_pairs, const int *modulus, const int *offset,
                    uint32_t *grid_out, uint32_t *adj_out, int *counts_out);

/* Runs `iterations` steps of the restated kernel. Arrays are per lattice cell
 * (x fastest), 19 doubles per cell; obstacle cells of out_pdfs are untouched.
 * lambda is the TRT magic parameter. */
int orc_run(int kernel, const int dims[3], const int periodic[3], const int *lattice,
            double omega, double lambda, double xforce, double rho_in, double rho_out,
            int iterations, int init_mode, const double *init_pdfs, double *out_pdfs,
            const int blk[3], int pad_mode);

/* One half (odd = 0: even step, 1: odd step) of a list AA step pair over
 * nodes [0, n_nodes) of f[d * n_cells + node] through the push adjacency adj
 * (n_nodes * 18), with the per-step body force added at the access that
 * follows each step; a complete pair equals orc_run's list AA pair bit for
 * bit. For checking decomposed (slab) layouts whose ghost nodes follow the
 * owned ones. */
int orc_list_aa_half(int odd, int n_nodes, int n_cells, const uint32_t *adj, double *f,
                     double omega, double lambda, double xforce);
/* The same half step over nodes [n0, n1) only (adj indexed by node). */
int orc_list_aa_half_range(int odd, int n0, int n1, int n_cells, const uint32_t *adj, double *f,
                           double omega, double lambda, double xforce);

/* The reference's -verify check (src/Kernel.c:451-625) on a field of logical
 * PDFs (same layout as orc_run's out_pdfs). Returns the L2 norm of the
 * relative error of the x-velocity profile at x = nX/2. */
double orc_verify_error(const int dims[3], const int *lattice, const double *pdfs, double omega, double xforce);

#ifdef __cplusplus
}
#endif

#endif
