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

/* Link words of the full-array AA layout: for every cell of the padded
 * (nX+2) x (nY+2) x pitch array, bit 31 = fluid cell, bit d = link d of the
 * cell does not reach a fluid node (wall or open face). Ghost and pad cells
 * get 0. cellOf(x,y,z) = (x+1)*xs + (y+1)*pitch + z + zoff. */
void lbmh_aa_links(const LatticeDesc *ld, int xs, int pitch, int zoff, uint32_t *link);
void lbmh_aa_links_range(const LatticeDesc *ld, int x0, int x1, int xs, int pitch, int zoff, uint32_t *link);

/* IEEE binary16 <-> binary32 (round to nearest even). */
float lbmh_f16_to_f32(uint16_t h);
uint16_t lbmh_f32_to_f16(float f);

/* Parses "v" or "a/b" into a double; returns 0 on success. */
int lbmh_parse_fraction(const char *s, double *out);

#ifdef __cplusplus
}
#endif

#endif
