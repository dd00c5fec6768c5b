/* lbm_host.h -- host-side layout builders of the B200 kernels (C).
 *
 * These produce exactly the reference's geometry masks, list numbering, SoA
 * padding and adjacency lists (bit for bit), plus the per-cell link words of
 * the full-array AA kernel.
 */
#ifndef LBM_HOST_H
#define LBM_HOST_H

#include <stdint.h>

#include "../../include/lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Cell index of the reference's lattice mask, x fastest (src/Lattice.h:60-76). */
static inline long lbmh_lidx(const int dims[3], int x, int y, int z)
{
	return ((long)z * dims[1] + y) * dims[0] + x;
}

/* nCells after SoA padding. padStr: NULL or "auto" (the reference default),
 * "no"/"off", or "m+o[,m+o]*" in bytes (src/Padding.c:19-244). Returns -1 and
 * prints a message for a malformed string. */
int lbmh_pad_cells(int nCells, int pdfBytes, const char *padStr);

/* Fluid-node numbering and adjacency for the push (list AA) or pull
 * (pull-split) propagation model. blk[3] = numbering blocks (0 = whole
 * extent). grid: nX*nY*nZ entries (obstacles get 0xffffffff); coords
 * (optional): 3 per node; adj: nFluid*18. Returns the node count. */
int lbmh_list_build(const LatticeDesc *ld, int pull, const int blk[3], int nCells,
                    uint32_t *grid, uint32_t *coords, uint32_t *adj);

/* One x-slab [x0, x1) of a list-AA (push adjacency) lattice split along x:
 * owned nodes (the slab's fluid cells, blocked numbering over the slab) then
 * ghost nodes (fluid cells of the neighbouring slabs that owned links
 * reach); adj indexes f[d * nCells + node] like lbmh_list_build's. Halo
 * lists per side (0: the x0 face, 1: the x1 - 1 face): ghost[side] = the
 * ghost slots that this slab's face cells reach through the face, own[side]
 * = the owned slots that the neighbour's face cells reach through it, both
 * in (z, y, link) order of the reaching cell, so that one slab's ghost list
 * and the neighbour's own list for their shared face pair up entry by entry. */
typedef struct {
	int L, nOwned, nGhost, nCells;
	uint32_t *grid;       /* L * nY * nZ slab cells (x fastest); obstacles 0xffffffff */
	uint32_t *adj;        /* nOwned * 18 */
	uint32_t *own[2], *ghost[2];
	long nOwnSlots[2], nGhostSlots[2];
} LbmhListSlab;

/* Builds the slab layout (halo[side] = 1: that face has a neighbour slab).
 * nCells: the owned and ghost nodes padded as the reference pads a list
 * (pad string, 8-byte PDFs) when quantum is 0, else rounded up to a multiple
 * of quantum (the reduced-storage layout's whole staging tiles).
 * Returns 0; -1 bad range (or a halo on a slab that spans the lattice);
 * -2 a link leaves through a face without a halo; -3 allocation failure;
 * -4 malformed padding string; -5 more PDFs than 32-bit indices address. */
int lbmh_list_slab_build(const LatticeDesc *ld, int x0, int x1, const int halo[2], const int blk[3],
                         const char *pad, int quantum, LbmhListSlab *s);
void lbmh_list_slab_free(LbmhListSlab *s);

/* The slab's inner tiles (of `tile` owned nodes): [*t0, *t1), a contiguous
 * range of tiles none of whose nodes links to a ghost node or owns a slot of
 * an own list, so that neither their even nor their odd step touches a slot
 * that a halo message carries. With the default numbering the
 * slab's two face planes are its first and last nodes and the range is the
 * rest; when face tiles are not all at the ends (blocked numbering), or
 * nothing is inner, the range is empty (0, 0). */
void lbmh_list_slab_inner_tiles(const LbmhListSlab *s, int tile, int *t0, int *t1);

/* Link words of the full-array AA layout: for every cell of the padded
 * (nX+2) x (nY+2) x pitch array, bit 31 = fluid cell, bit d = link d of the
 * cell does not reach a fluid node (wall or open face). Ghost and pad cells
 * get 0. cellOf(x,y,z) = (x+1)*xs + (y+1)*pitch + z + zoff. */
void lbmh_aa_links(const LatticeDesc *ld, int xs, int pitch, int zoff, uint32_t *link);
void lbmh_aa_links_range(const LatticeDesc *ld, int x0, int x1, int xs, int pitch, int zoff, uint32_t *link);

/* IEEE binary16 <-> binary32 (round to nearest even). */
/* Profile error of an x-velocity slice (nY x nZ, slice[y * nz + z]) against
 * the analytic channel profile, and with write_file the reference's
 * flow-profile.dat (src/Kernel.c:547-616). */
double lbmh_verify_profile(int ny, int nz, double omega, double xforce, const double *slice, int write_file);

float lbmh_f16_to_f32(uint16_t h);
uint16_t lbmh_f32_to_f16(float f);

/* Parses "v" or "a/b" into a double; returns 0 on success. */
int lbmh_parse_fraction(const char *s, double *out);

#ifdef __cplusplus
}
#endif

#endif
