/* lbm_host.c -- host side of the B200 D3Q19 kernels: geometry masks, list
 * numbering/padding/adjacency, AA link words, and the reference's host
 * helpers (initial density/velocity, Poiseuille check, mean density) that
 * operate through a kernel's GetNode/SetNode.
 *
 * Semantics follow the reference exactly (masks, numbering and adjacency are
 * compared bit for bit by the tests); see each function for the reference
 * lines it reproduces.
 */
#include "lbm_host.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <sys/stat.h>

/* D3Q19 velocity set in the reference's order N,S,E,W,NE,SE,NW,SW,T,TN,TE,
 * TW,TS,B,BS,BN,BW,BE,C (src/Kernel.h:121-140): {cx, cy, cz, inverse}. */
static const struct { int x, y, z, inv; } kVel[19] = {
	{ 0, 1, 0, 1}, { 0,-1, 0, 0}, { 1, 0, 0, 3}, {-1, 0, 0, 2},
	{ 1, 1, 0, 7}, { 1,-1, 0, 6}, {-1, 1, 0, 5}, {-1,-1, 0, 4},
	{ 0, 0, 1,13}, { 0, 1, 1,14}, { 1, 0, 1,16}, {-1, 0, 1,17}, { 0,-1, 1,15},
	{ 0, 0,-1, 8}, { 0,-1,-1, 9}, { 0, 1,-1,12}, {-1, 0,-1,10}, { 1, 0,-1,11},
	{ 0, 0, 0,18}
};
enum { dN, dS, dE, dW, dNE, dSE, dNW, dSW, dT, dTN, dTE, dTW, dTS, dB, dBS, dBN, dBW, dBE, dC };

/* ------------------------------------------------------------------------ */
/* Geometry: GeoCreateByStr / GeoCreateByType (src/Geometry.c:37-281). */

static const char *kGeoNames[] = { "box", "channel", "pipe", "blocks", "fluid" };

int lbm_geo_spheres(const int dims[3], uint64_t seed, double porosity, double rmin, double rmax,
                    int rsaAttempts, LatticeDesc *ld, double *stats);

int lbm_geo_create(const char *geo, int dims[3], int periodic[3], LatticeDesc *ld)
{
	int type, block = 8;
	if (!strncasecmp("channel", geo, 7)) type = 1;
	else if (!strncasecmp("box", geo, 3)) type = 0;
	else if (!strncasecmp("pipe", geo, 4)) type = 2;
	else if (!strncasecmp("blocks", geo, 6)) {
		type = 3;
		if (strlen(geo) > 7) block = atoi(geo + 7);
		int dmin = dims[0] < dims[1] ? dims[0] : dims[1];
		if (dims[2] < dmin) dmin = dims[2];
		if (block < 0 || (block > 0 && block > dmin / 2)) {
			printf("ERROR: block size for geometry must be > 0 and smaller than half of the smalest dimension.\n");
			return -1;
		}
	}
	else if (!strncasecmp("fluid", geo, 5)) type = 4;
	else if (!strncasecmp("spheres", geo, 7)) {
		/* spheres:<seed>:<porosity>:<rmin>:<rmax> (defaults 1:0.4:6:12) */
		unsigned long long seed = 1;
		double por = 0.4, rmin = 6.0, rmax = 12.0;
		if (geo[7] == ':') sscanf(geo + 8, "%llu:%lf:%lf:%lf", &seed, &por, &rmin, &rmax);
		return lbm_geo_spheres(dims, (uint64_t)seed, por, rmin, rmax, 20000, ld, NULL);
	}
	else {
		printf("ERROR: unknown geometry specified.\n");
		return -1;
	}

	const int nx = dims[0], ny = dims[1], nz = dims[2];
	const long n = (long)nx * ny * nz;

	ld->Dims[0] = nx; ld->Dims[1] = ny; ld->Dims[2] = nz;
	ld->nCells = (int)n;
	/* recorded before the geometry forces its own periodicity (the kernels
	 * see the caller's flags, src/Geometry.c:115-139) */
	ld->PeriodicX = periodic[0]; ld->PeriodicY = periodic[1]; ld->PeriodicZ = periodic[2];
	ld->Name = kGeoNames[type];

	LatticeT *lat = (LatticeT *)malloc(sizeof(LatticeT) * (size_t)n);
	if (!lat) { printf("ERROR: allocating the lattice mask failed.\n"); return -1; }
	ld->Lattice = lat;
	for (long i = 0; i < n; ++i) lat[i] = LAT_CELL_FLUID;

	if (type == 1 || type == 2 || type == 3) periodic[0] = 1;
	else if (type == 4) periodic[0] = periodic[1] = periodic[2] = 1;

	/* boundary planes, x then y then z: later planes win on shared edges */
	for (int axis = 0; axis < 3; ++axis) {
		const LatticeT v = periodic[axis] ? LAT_CELL_FLUID : LAT_CELL_OBSTACLE;
		const int na = dims[axis];
		for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
			const int c = axis == 0 ? x : (axis == 1 ? y : z);
			if (c == 0 || c == na - 1) lat[lbmh_lidx(dims, x, y, z)] = v;
		}
	}

	if (type == 2) {
		const double czc = nz / 2.0 - 0.5, cyc = ny / 2.0 - 0.5;
		const double diam = ny < nz ? ny : nz;
		const double rr = (diam / 2 - 1) * (diam / 2 - 1);
		for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) {
			const double r2 = (z - czc) * (z - czc) + (y - cyc) * (y - cyc);
			if (r2 < rr) continue;
			for (int x = 0; x < nx; ++x) lat[lbmh_lidx(dims, x, y, z)] = LAT_CELL_OBSTACLE;
		}
	}
	else if (type == 3 && block > 0) {
		const int b2 = 2 * block;
		for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
			if (z % b2 >= block && y % b2 >= block && x % b2 >= block)
				lat[lbmh_lidx(dims, x, y, z)] = LAT_CELL_OBSTACLE;
		}
	}

	ld->nObst = ld->nFluid = ld->nInlet = ld->nOutlet = 0;
	for (long i = 0; i < n; ++i) {
		switch (lat[i]) {
			case LAT_CELL_OBSTACLE: ld->nObst++; break;
			case LAT_CELL_INLET:    ld->nInlet++; ld->nFluid++; break;
			case LAT_CELL_OUTLET:   ld->nOutlet++; ld->nFluid++; break;
			default:                ld->nFluid++; break;
		}
	}
	return 0;
}

/* ------------------------------------------------------------------------ */
/* SoA padding (src/Padding.c:19-244). */

int lbmh_pad_cells(int nCells, int pdfBytes, const char *padStr)
{
	int mods[64], offs[64], k = 0;
	if (padStr == NULL || !strncmp(padStr, "auto", 4)) {
		mods[0] = 2 * 1024 * 1024 * 8; offs[0] = 2 * 1024 * 1024 + 512; /* 2 MiB TLB pages */
		mods[1] = 256 * 64;            offs[1] = 128;                   /* L2, 256 sets */
		k = 2;
	}
	else if (!strncmp(padStr, "no", 2) || !strncmp(padStr, "off", 3)) {
		k = 0;
	}
	else {
		const char *s = padStr;
		while (*s) {
			char *end;
			long m = strtol(s, &end, 10);
			if (end == s || *end != '+' || m < 0) { printf("ERROR: malformed padding string \"%s\".\n", padStr); return -1; }
			s = end + 1;
			long o = strtol(s, &end, 10);
			if (end == s || o < 0 || (*end != ',' && *end != 0)) { printf("ERROR: malformed padding string \"%s\".\n", padStr); return -1; }
			if (o >= m && m != 0) { printf("ERROR: offset in padding entry %d is equal or larger than modulus.\n", k); return -1; }
			if (k == 64) { printf("ERROR: too many padding entries.\n"); return -1; }
			mods[k] = (int)m; offs[k] = (int)o; ++k;
			s = *end ? end + 1 : end;
		}
	}
	for (int i = 0; i < k; ++i) {
		int pad;
		if (mods[i] == 0) {
			pad = offs[i] * pdfBytes; /* the reference multiplies here (Padding.c:223) */
		}
		else {
			const int modCells = mods[i] / pdfBytes;
			if (modCells == 0) { printf("ERROR: modulus of %d byte in padding entry %d becomes zero.\n", mods[i], i); return -1; }
			pad = (offs[i] / pdfBytes + modCells - nCells % modCells) % modCells;
		}
		nCells += pad;
	}
	return nCells;
}

/* ------------------------------------------------------------------------ */
/* List numbering and adjacency (src/BenchKernelD3Q19ListAaPvCommon.c:587-792,
 * src/BenchKernelD3Q19ListPullSplitNtCommon.c:548-755). */

int lbmh_list_build(const LatticeDesc *ld, int pull, const int blk[3], int nCells,
                    uint32_t *grid, uint32_t *coords, uint32_t *adj)
{
	const int *dims = ld->Dims;
	const int nx = dims[0], ny = dims[1], nz = dims[2];
	const long n = (long)nx * ny * nz;
	int bx = blk && blk[0] > 0 ? blk[0] : nx;
	int by = blk && blk[1] > 0 ? blk[1] : ny;
	int bz = blk && blk[2] > 0 ? blk[2] : nz;

	for (long i = 0; i < n; ++i) grid[i] = 0xffffffffu;

	/* blocked numbering, x -> y -> z with z innermost */
	uint32_t count = 0;
	for (int x0 = 0; x0 < nx; x0 += bx)
	for (int y0 = 0; y0 < ny; y0 += by)
	for (int z0 = 0; z0 < nz; z0 += bz) {
		const int x1 = x0 + bx < nx ? x0 + bx : nx;
		const int y1 = y0 + by < ny ? y0 + by : ny;
		const int z1 = z0 + bz < nz ? z0 + bz : nz;
		for (int x = x0; x < x1; ++x)
		for (int y = y0; y < y1; ++y)
		for (int z = z0; z < z1; ++z) {
			const long li = lbmh_lidx(dims, x, y, z);
			if (ld->Lattice[li] == LAT_CELL_OBSTACLE) continue;
			grid[li] = count;
			if (coords) { coords[3 * (long)count] = x; coords[3 * (long)count + 1] = y; coords[3 * (long)count + 2] = z; }
			++count;
		}
	}

	const int per[3] = { ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ };
	const int sign = pull ? -1 : 1;
	const uint32_t nc = (uint32_t)nCells;

	/* walk the nodes in numbering order again to fill the adjacency */
	for (int x0 = 0; x0 < nx; x0 += bx)
	for (int y0 = 0; y0 < ny; y0 += by)
	for (int z0 = 0; z0 < nz; z0 += bz) {
		const int x1 = x0 + bx < nx ? x0 + bx : nx;
		const int y1 = y0 + by < ny ? y0 + by : ny;
		const int z1 = z0 + bz < nz ? z0 + bz : nz;
		for (int x = x0; x < x1; ++x)
		for (int y = y0; y < y1; ++y)
		for (int z = z0; z < z1; ++z) {
			const long li = lbmh_lidx(dims, x, y, z);
			if (ld->Lattice[li] == LAT_CELL_OBSTACLE) continue;
			const uint32_t self = grid[li];
			uint32_t *row = adj + (long)self * 18;
			for (int d = 0; d < 18; ++d) {
				int q[3] = { x + sign * kVel[d].x, y + sign * kVel[d].y, z + sign * kVel[d].z };
				int out = 0, crossPer = 0;
				for (int a = 0; a < 3; ++a) {
					const int o = q[a] < 0 || q[a] >= dims[a];
					out |= o;
					crossPer |= o && per[a];
				}
				uint32_t dst = (uint32_t)kVel[d].inv * nc + self; /* bounce back by default */
				if (crossPer) {
					/* every crossed axis wraps once a periodic one is crossed */
					for (int a = 0; a < 3; ++a) q[a] = q[a] < 0 ? dims[a] - 1 : (q[a] >= dims[a] ? 0 : q[a]);
					out = 0;
				}
				if (!out) {
					const long nb = lbmh_lidx(dims, q[0], q[1], q[2]);
					if (ld->Lattice[nb] != LAT_CELL_OBSTACLE) dst = (uint32_t)d * nc + grid[nb];
				}
				row[d] = dst;
			}
		}
	}
	return (int)count;
}

/* ------------------------------------------------------------------------ */
/* One x-slab [x0, x1) of a list-AA lattice split along x (no counterpart in
 * the reference, whose list kernels address one array). Owned nodes are the
 * slab's fluid cells in lbmh_list_build's blocked numbering over the slab;
 * ghost nodes follow them: the fluid cells of the neighbouring slabs that an
 * owned node's link reaches, in the order the owned nodes first reach them.
 * Links follow the whole lattice's rule, so an owned node's adjacency equals
 * its adjacency in the undivided lattice with remote nodes replaced by ghosts. */

/* Target of link d (push model) of fluid cell (x, y, z) under the rule of
 * lbmh_list_build: 1 and the cell in q if the link reaches a fluid cell, 0 if
 * it bounces back. */
static int list_link_target(const LatticeDesc *ld, int x, int y, int z, int d, int q[3])
{
	const int *dims = ld->Dims;
	const int per[3] = { ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ };
	q[0] = x + kVel[d].x; q[1] = y + kVel[d].y; q[2] = z + kVel[d].z;
	int out = 0, crossPer = 0;
	for (int a = 0; a < 3; ++a) {
		const int o = q[a] < 0 || q[a] >= dims[a];
		out |= o;
		crossPer |= o && per[a];
	}
	if (crossPer) {
		for (int a = 0; a < 3; ++a) q[a] = q[a] < 0 ? dims[a] - 1 : (q[a] >= dims[a] ? 0 : q[a]);
		out = 0;
	}
	if (out) return 0;
	return ld->Lattice[lbmh_lidx(dims, q[0], q[1], q[2])] != LAT_CELL_OBSTACLE;
}

void lbmh_list_slab_free(LbmhListSlab *s)
{
	free(s->grid); free(s->adj);
	for (int k = 0; k < 2; ++k) { free(s->own[k]); free(s->ghost[k]); }
	memset(s, 0, sizeof(*s));
}

/* Visits the slab's fluid cells in the owned numbering order. */
#define SLAB_CELLS_BEGIN(ld, x0, x1, bx, by, bz)                                   \
	for (int X0 = (x0); X0 < (x1); X0 += (bx))                                     \
	for (int Y0 = 0; Y0 < (ld)->Dims[1]; Y0 += (by))                               \
	for (int Z0 = 0; Z0 < (ld)->Dims[2]; Z0 += (bz)) {                             \
		const int X1 = X0 + (bx) < (x1) ? X0 + (bx) : (x1);                        \
		const int Y1 = Y0 + (by) < (ld)->Dims[1] ? Y0 + (by) : (ld)->Dims[1];      \
		const int Z1 = Z0 + (bz) < (ld)->Dims[2] ? Z0 + (bz) : (ld)->Dims[2];      \
		for (int x = X0; x < X1; ++x)                                              \
		for (int y = Y0; y < Y1; ++y)                                              \
		for (int z = Z0; z < Z1; ++z) {                                            \
			if ((ld)->Lattice[lbmh_lidx((ld)->Dims, x, y, z)] == LAT_CELL_OBSTACLE) continue;
#define SLAB_CELLS_END }}

int lbmh_list_slab_build(const LatticeDesc *ld, int x0, int x1, const int halo[2], const int blk[3],
                         const char *pad, int quantum, LbmhListSlab *s)
{
	const int nx = ld->Dims[0], ny = ld->Dims[1], nz = ld->Dims[2];
	const int L = x1 - x0;
	memset(s, 0, sizeof(*s));
	if (x0 < 0 || x1 > nx || L < 1) return -1;
	if ((halo[0] || halo[1]) && L == nx) return -1;
	const int bx = blk && blk[0] > 0 ? blk[0] : L;
	const int by = blk && blk[1] > 0 ? blk[1] : ny;
	const int bz = blk && blk[2] > 0 ? blk[2] : nz;
	const long plane = (long)ny * nz;
	const int xLo = (x0 - 1 + nx) % nx, xHi = x1 % nx;
	s->L = L;
	s->grid = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)L * plane);
	int *gmap[2];
	gmap[0] = (int *)malloc(sizeof(int) * (size_t)plane);
	gmap[1] = xHi == xLo ? gmap[0] : (int *)malloc(sizeof(int) * (size_t)plane);
	int rc = 0;
	if (!s->grid || !gmap[0] || !gmap[1]) { rc = -3; goto done; }
	for (long i = 0; i < (long)L * plane; ++i) s->grid[i] = 0xffffffffu;
	for (long i = 0; i < plane; ++i) gmap[0][i] = gmap[1][i] = -1;
	const int ldims[3] = { L, ny, nz };

	uint32_t count = 0;
	SLAB_CELLS_BEGIN(ld, x0, x1, bx, by, bz)
		s->grid[lbmh_lidx(ldims, x - x0, y, z)] = count++;
	SLAB_CELLS_END
	s->nOwned = (int)count;

	/* ghosts, in the order the owned nodes first reach them */
	int nGhost = 0;
	SLAB_CELLS_BEGIN(ld, x0, x1, bx, by, bz)
		for (int d = 0; d < 18; ++d) {
			int q[3];
			if (!list_link_target(ld, x, y, z, d, q) || (q[0] >= x0 && q[0] < x1)) continue;
			const int side = kVel[d].x < 0 ? 0 : 1;
			if (!halo[side]) { rc = -2; goto done; }
			int *g = &gmap[side][(long)q[2] * ny + q[1]];
			if (*g < 0) *g = nGhost++;
		}
	SLAB_CELLS_END
	s->nGhost = nGhost;
	if (quantum > 0) {
		const long n = s->nOwned + nGhost > 0 ? s->nOwned + nGhost : 1;
		s->nCells = (int)((n + quantum - 1) / quantum * quantum);
	} else {
		s->nCells = lbmh_pad_cells(s->nOwned + nGhost, (int)sizeof(double), pad);
	}
	if (s->nCells < 0) { rc = -4; goto done; }
	if ((uint64_t)19 * (uint64_t)s->nCells >= (1ull << 32)) { rc = -5; goto done; }
	const uint32_t nc = (uint32_t)s->nCells;

	s->adj = (uint32_t *)malloc(sizeof(uint32_t) * 18 * (size_t)(s->nOwned > 0 ? s->nOwned : 1));
	if (!s->adj) { rc = -3; goto done; }
	SLAB_CELLS_BEGIN(ld, x0, x1, bx, by, bz)
		const uint32_t self = s->grid[lbmh_lidx(ldims, x - x0, y, z)];
		uint32_t *row = s->adj + (size_t)self * 18;
		for (int d = 0; d < 18; ++d) {
			int q[3];
			uint32_t dst = (uint32_t)kVel[d].inv * nc + self; /* bounce back */
			if (list_link_target(ld, x, y, z, d, q)) {
				if (q[0] >= x0 && q[0] < x1)
					dst = (uint32_t)d * nc + s->grid[lbmh_lidx(ldims, q[0] - x0, q[1], q[2])];
				else
					dst = (uint32_t)d * nc + (uint32_t)(s->nOwned + gmap[kVel[d].x < 0 ? 0 : 1][(long)q[2] * ny + q[1]]);
			}
			row[d] = dst;
		}
	SLAB_CELLS_END

	/* halo slot lists. Side 0 faces x0, side 1 faces x1 - 1. ghost[side]:
	 * the ghost slots this slab's face cells reach through that face; own[side]:
	 * the owned slots the neighbour's face cells reach through it. Both are
	 * in the order (z, y, d) of the reaching cell and link, so a slab's ghost
	 * list and its neighbour's own list for the shared face match entry for
	 * entry. */
	for (int side = 0; side < 2; ++side) {
		if (!halo[side]) continue;
		s->ghost[side] = (uint32_t *)malloc(sizeof(uint32_t) * 5 * (size_t)plane);
		s->own[side] = (uint32_t *)malloc(sizeof(uint32_t) * 5 * (size_t)plane);
		if (!s->ghost[side] || !s->own[side]) { rc = -3; goto done; }
		const int xf = side ? x1 - 1 : x0;        /* this slab's face plane */
		const int xn = side ? xHi : xLo;          /* the neighbour's face plane */
		const int toward = side ? 1 : -1;
		long ng = 0, no = 0;
		for (int z = 0; z < nz; ++z)
		for (int y = 0; y < ny; ++y) {
			if (ld->Lattice[lbmh_lidx(ld->Dims, xf, y, z)] != LAT_CELL_OBSTACLE)
				for (int d = 0; d < 18; ++d) {
					int q[3];
					if (kVel[d].x != toward || !list_link_target(ld, xf, y, z, d, q)) continue;
					if (q[0] >= x0 && q[0] < x1) continue;
					s->ghost[side][ng++] = (uint32_t)d * nc + (uint32_t)(s->nOwned + gmap[side][(long)q[2] * ny + q[1]]);
				}
			if (ld->Lattice[lbmh_lidx(ld->Dims, xn, y, z)] != LAT_CELL_OBSTACLE)
				for (int d = 0; d < 18; ++d) {
					int q[3];
					if (kVel[d].x != -toward || !list_link_target(ld, xn, y, z, d, q)) continue;
					if (q[0] < x0 || q[0] >= x1) continue;
					s->own[side][no++] = (uint32_t)d * nc + s->grid[lbmh_lidx(ldims, q[0] - x0, q[1], q[2])];
				}
		}
		s->nGhostSlots[side] = ng;
		s->nOwnSlots[side] = no;
	}
done:
	if (gmap[1] != gmap[0]) free(gmap[1]);
	free(gmap[0]);
	if (rc) lbmh_list_slab_free(s);
	return rc;
}

void lbmh_list_slab_inner_tiles(const LbmhListSlab *s, int tile, int *t0, int *t1)
{
	const int nOwned = s->nOwned;
	const int nTiles = (nOwned + tile - 1) / tile;
	/* a tile is inner when none of its nodes links to a ghost node and no
	 * slot of its nodes is in an own list (a slot the neighbour reads and
	 * writes) */
	int lead = 0, trail = 0, inner = 1;
	char *face = (char *)calloc(nTiles > 0 ? nTiles : 1, 1);
	if (!face) { *t0 = *t1 = 0; return; }
	for (long n = 0; n < nOwned; ++n)
		for (int d = 0; d < 18; ++d)
			if ((int)(s->adj[n * 18 + d] % (uint32_t)s->nCells) >= nOwned) { face[n / tile] = 1; break; }
	for (int side = 0; side < 2; ++side)
		for (long k = 0; s->own[side] && k < s->nOwnSlots[side]; ++k)
			face[(s->own[side][k] % (uint32_t)s->nCells) / tile] = 1;
	while (lead < nTiles && face[lead]) ++lead;
	while (trail < nTiles - lead && face[nTiles - 1 - trail]) ++trail;
	for (int t = lead; t < nTiles - trail; ++t) inner &= !face[t];
	free(face);
	if (!inner || lead >= nTiles - trail) { *t0 = *t1 = 0; return; }
	*t0 = lead;
	*t1 = nTiles - trail;
}

/* ------------------------------------------------------------------------ */
/* AA link words. A link d of fluid cell x is "reversed" when x + c_d is not a
 * fluid node reached directly or through a periodic wrap: an obstacle inside
 * the domain, an obstacle reached through a wrap, or a non-periodic exit. The
 * classification matches the reference's fix-up list construction
 * (src/BenchKernelD3Q19AaCommon.c:512-621). */

void lbmh_aa_links(const LatticeDesc *ld, int xs, int pitch, int zoff, uint32_t *link)
{
	lbmh_aa_links_range(ld, 0, ld->Dims[0], xs, pitch, zoff, link);
}

/* The link words of the x-slab [x0, x1) of the lattice ld, in the slab's own
 * full-array layout (local x = global x - x0): the classification uses the
 * whole lattice, so a link into a neighbouring slab is reversed exactly when
 * the global neighbour is not a fluid node. */
void lbmh_aa_links_range(const LatticeDesc *ld, int x0, int x1, int xs, int pitch, int zoff, uint32_t *link)
{
	const int *dims = ld->Dims;
	const int ny = dims[1], nz = dims[2];
	const int per[3] = { ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ };
	const long total = (long)(x1 - x0 + 2) * xs;
	memset(link, 0, sizeof(uint32_t) * (size_t)total);

	for (int x = x0; x < x1; ++x) for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) {
		if (ld->Lattice[lbmh_lidx(dims, x, y, z)] == LAT_CELL_OBSTACLE) continue;
		uint32_t w = 0x80000000u;
		for (int d = 0; d < 18; ++d) {
			int q[3] = { x + kVel[d].x, y + kVel[d].y, z + kVel[d].z };
			int out = 0, crossPer = 0;
			for (int a = 0; a < 3; ++a) {
				const int o = q[a] < 0 || q[a] >= dims[a];
				out |= o;
				crossPer |= o && per[a];
			}
			int reversed;
			if (crossPer) {
				for (int a = 0; a < 3; ++a) q[a] = q[a] < 0 ? dims[a] - 1 : (q[a] >= dims[a] ? 0 : q[a]);
				reversed = ld->Lattice[lbmh_lidx(dims, q[0], q[1], q[2])] == LAT_CELL_OBSTACLE;
			}
			else if (out) {
				reversed = 1; /* open face */
			}
			else {
				reversed = ld->Lattice[lbmh_lidx(dims, q[0], q[1], q[2])] == LAT_CELL_OBSTACLE;
			}
			if (reversed) w |= 1u << d;
		}
		link[(long)(x - x0 + 1) * xs + (long)(y + 1) * pitch + z + zoff] = w;
	}
}

int lbmh_parse_fraction(const char *s, double *out)
{
	char *end;
	double a = strtod(s, &end);
	if (end == s) return -1;
	if (*end == '/') {
		const char *t = end + 1;
		double b = strtod(t, &end);
		if (end == t || b == 0.0 || *end) return -1;
		*out = a / b;
		return 0;
	}
	if (*end) return -1;
	*out = a;
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Reference host helpers through GetNode/SetNode (src/Kernel.c). */

/* f_i as KernelSetInitialDensity writes it (src/Kernel.c:276-332): the
 * equilibrium scaled by omega (the reference's own formula). */
static void ref_init_pdfs(double omega, double dens, double ux, double uy, double uz, double *p)
{
	const double w0 = 1.0 / 3.0, w1 = 1.0 / 18.0, w2 = 1.0 / 36.0;
	const double a0 = 3.0 * w0 * omega, a1 = 3.0 * w1 * omega, a2 = 3.0 * w2 * omega;
	const double third = 1.0 / 3.0;
	const double t = third * dens - 0.5 * (ux * ux + uy * uy + uz * uz);
	const double xmy = ux - uy, xpy = ux + uy, xmz = ux - uz, xpz = ux + uz, ymz = uy - uz, ypz = uy + uz;
	p[dC]  = a0 * (t);
	p[dNW] = a2 * (t - xmy + 1.5 * (xmy * xmy));
	p[dSE] = a2 * (t + xmy + 1.5 * (xmy * xmy));
	p[dNE] = a2 * (t + xpy + 1.5 * (xpy * xpy));
	p[dSW] = a2 * (t - xpy + 1.5 * (xpy * xpy));
	p[dTW] = a2 * (t - xmz + 1.5 * (xmz * xmz));
	p[dBE] = a2 * (t + xmz + 1.5 * (xmz * xmz));
	p[dTE] = a2 * (t + xpz + 1.5 * (xpz * xpz));
	p[dBW] = a2 * (t - xpz + 1.5 * (xpz * xpz));
	p[dTS] = a2 * (t - ymz + 1.5 * (ymz * ymz));
	p[dBN] = a2 * (t + ymz + 1.5 * (ymz * ymz));
	p[dTN] = a2 * (t + ypz + 1.5 * (ypz * ypz));
	p[dBS] = a2 * (t - ypz + 1.5 * (ypz * ypz));
	p[dN]  = a1 * (t + uy + 1.5 * (uy * uy));
	p[dS]  = a1 * (t - uy + 1.5 * (uy * uy));
	p[dE]  = a1 * (t + ux + 1.5 * (ux * ux));
	p[dW]  = a1 * (t - ux + 1.5 * (ux * ux));
	p[dT]  = a1 * (t + uz + 1.5 * (uz * uz));
	p[dB]  = a1 * (t - uz + 1.5 * (uz * uz));
}

void lbm_set_initial_density(LatticeDesc *ld, KernelData *kd, CaseData *cd)
{
	const int *dims = ld->Dims;
	double p[19];
	for (int z = 0; z < dims[2]; ++z) for (int y = 0; y < dims[1]; ++y) for (int x = 0; x < dims[0]; ++x) {
		if (ld->Lattice[lbmh_lidx(dims, x, y, z)] == LAT_CELL_OBSTACLE) continue;
		const double dens = cd->RhoIn + (cd->RhoOut - cd->RhoIn) * (x) / (dims[0] - 1.0);
		ref_init_pdfs(cd->Omega, dens, 0.0, 0.0, 0.0, p);
		kd->SetNode(kd, x, y, z, p);
	}
}

void lbm_set_initial_velocity(LatticeDesc *ld, KernelData *kd, CaseData *cd)
{
	/* src/Kernel.c:344-438: uses a density of 1 and zero velocity */
	const int *dims = ld->Dims;
	double p[19];
	for (int z = 0; z < dims[2]; ++z) for (int y = 0; y < dims[1]; ++y) for (int x = 0; x < dims[0]; ++x) {
		if (ld->Lattice[lbmh_lidx(dims, x, y, z)] != LAT_CELL_FLUID) continue;
		ref_init_pdfs(cd->Omega, 1.0, 0.0, 0.0, 0.0, p);
		kd->SetNode(kd, x, y, z, p);
	}
}

double lbm_density(KernelData *kd, LatticeDesc *ld)
{
	const int *dims = ld->Dims;
	double p[19], sum = 0.0;
	for (int z = 0; z < dims[2]; ++z) for (int y = 0; y < dims[1]; ++y) for (int x = 0; x < dims[0]; ++x) {
		if (ld->Lattice[lbmh_lidx(dims, x, y, z)] == LAT_CELL_OBSTACLE) continue;
		kd->GetNode(kd, x, y, z, p);
		double local = 0.0;
		for (int d = 0; d < 19; ++d) local += p[d];
		sum += local;
	}
	return sum / ld->nFluid;
}

static double x_velocity(const double *p)
{
	return p[dE] + p[dNE] + p[dSE] + p[dTE] + p[dBE] - p[dW] - p[dNW] - p[dSW] - p[dTW] - p[dBW];
}

/* The profile error of an x-velocity slice (slice[y * nz + z]) and, with
 * write_file, the reference's flow-profile.dat (src/Kernel.c:547-616). */
double lbmh_verify_profile(int ny, int nz, double omega, double xforce, const double *slice, int write_file)
{
	const double visc = (1.0 / omega - 0.5) / 3.0;
	const int evenNy = ny % 2 == 0;
	const int ym = (ny - evenNy - 1) / 2;
	const double center = ny / 2.0;
	const double rmax = (double)ny / 2.0 - 1.0;
	const double r2max = rmax * rmax;
	const double umax = xforce * r2max / (2.0 * visc);

	FILE *fh = NULL;
	if (write_file) {
		fh = fopen("flow-profile.dat", "w");
		if (fh) fprintf(fh, "# z coord., radius, analytic, simulation, diff abs, diff rel, undim_analytic, undim_sim\n");
	}
	double dev = 0.0;
	for (int z = 0; z < nz; ++z) {
		const double r = z - center + 0.5;
		const double r2 = r * r;
		const double ua = r2 >= r2max ? 0.0 : xforce * (r2max - r2) / (2.0 * visc);
		const double us = evenNy ? (slice[ym * nz + z] + slice[(ym + 1) * nz + z]) / 2.0 : slice[ym * nz + z];
		double rel = 0.0;
		if (ua != 0.0) {
			rel = fabs(ua - us) / ua;
			dev += rel * rel;
		}
		if (fh) fprintf(fh, "%d\t%e\t%e\t%e\t%e\t%e\t%e\t%e\n", z, r / center, ua, us, fabs(ua - us), rel, ua / umax, us / umax);
	}
	if (fh) fclose(fh);
	return sqrt(dev);
}

double lbm_verify(LatticeDesc *ld, KernelData *kd, CaseData *cd, int write_file)
{
	const int nx = ld->Dims[0], ny = ld->Dims[1], nz = ld->Dims[2];
	const int xs = nx / 2;
	double *slice = (double *)malloc(sizeof(double) * (size_t)ny * nz);
	double p[19];

	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) {
		double u = 0.0;
		if (ld->Lattice[lbmh_lidx(ld->Dims, xs, y, z)] != LAT_CELL_OBSTACLE) {
			kd->GetNode(kd, xs, y, z, p);
			u = x_velocity(p);
			u += 0.5 * cd->XForce;
		}
		slice[y * nz + z] = u;
	}
	const double err = lbmh_verify_profile(ny, nz, cd->Omega, cd->XForce, slice, write_file);
	free(slice);
	return err;
}

/* ------------------------------------------------------------------------ */
/* Legacy VTK dump of one state, the file format of the reference's VtkWrite
 * (src/Vtk.c:51-245): STRUCTURED_POINTS header, then three binary blocks in
 * cell order x fastest -- the cell flags as unsigned char, the density
 * sum_i f_i and the velocity (sum_i c_i f_i, plus F/2 along x: the form of
 * the reference's VERIFICATION builds, whose body force these kernels always
 * apply) as big-endian doubles, 0 at obstacles. The sums run in the
 * reference's order, so an FP64 state that is bit-identical gives a file that
 * is byte-identical. */

static void vtk_put_be64(FILE *fh, double v)
{
	uint64_t u;
	unsigned char b[8];
	memcpy(&u, &v, 8);
	for (int k = 0; k < 8; ++k) b[k] = (unsigned char)(u >> (56 - 8 * k));
	fwrite(b, 1, 8, fh);
}

int lbm_vtk_write_file(LatticeDesc *ld, KernelData *kd, CaseData *cd, int iteration, const char *path)
{
	const int nx = ld->Dims[0], ny = ld->Dims[1], nz = ld->Dims[2];
	FILE *fh = fopen(path, "w");
	if (!fh) return -1;
	fprintf(fh, "# vtk DataFile Version 1.0\n");
	fprintf(fh, "Comment: lid driven cavity, iteration % 4d\n", iteration);
	fprintf(fh, "BINARY\n");
	fprintf(fh, "DATASET STRUCTURED_POINTS\n");
	fprintf(fh, "DIMENSIONS %d %d %d\n", nx, ny, nz);
	fprintf(fh, "ORIGIN 0 0 0 \n");
	fprintf(fh, "SPACING 1 1 1\n");
	fprintf(fh, "POINT_DATA %d\n", nx * ny * nz);

	fprintf(fh, "SCALARS NodesTypes unsigned_char 1\n");
	fprintf(fh, "LOOKUP_TABLE default\n");
	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
		unsigned char c = (unsigned char)ld->Lattice[lbmh_lidx(ld->Dims, x, y, z)];
		fwrite(&c, 1, 1, fh);
	}

	double p[19];
	fprintf(fh, "SCALARS Density double\n");
	fprintf(fh, "LOOKUP_TABLE default\n");
	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
		double rho = 0.0;
		if (ld->Lattice[lbmh_lidx(ld->Dims, x, y, z)] != LAT_CELL_OBSTACLE) {
			kd->GetNode(kd, x, y, z, p);
			for (int d = 0; d < 19; ++d) rho += p[d];
		}
		vtk_put_be64(fh, rho);
	}

	fprintf(fh, "VECTORS VelocityVectors double\n");
	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
		double ux = 0.0, uy = 0.0, uz = 0.0;
		if (ld->Lattice[lbmh_lidx(ld->Dims, x, y, z)] != LAT_CELL_OBSTACLE) {
			kd->GetNode(kd, x, y, z, p);
			ux = x_velocity(p);
			uy = p[dN] + p[dNE] + p[dNW] + p[dTN] + p[dBN] - p[dS] - p[dSE] - p[dSW] - p[dTS] - p[dBS];
			uz = p[dT] + p[dTE] + p[dTW] + p[dTN] + p[dTS] - p[dB] - p[dBE] - p[dBW] - p[dBN] - p[dBS];
			ux += 0.5 * cd->XForce;
		}
		vtk_put_be64(fh, ux);
		vtk_put_be64(fh, uy);
		vtk_put_be64(fh, uz);
	}
	return fclose(fh) == 0 ? 0 : -1;
}

int lbm_vtk_write(LatticeDesc *ld, KernelData *kd, CaseData *cd, int iteration)
{
	struct stat st;
	if (stat("vtk", &st) != 0) {
		if (mkdir("vtk", 0700) != 0) {
			printf("ERROR: cannot create directory vtk.\n");
			return -1;
		}
		printf("# created directory vtk.\n");
	} else if (!S_ISDIR(st.st_mode)) {
		printf("ERROR: cannot create subdirectory vtk as already a file with the same name exists.\n");
		return -1;
	}
	char name[64];
	snprintf(name, sizeof(name), "vtk/file-%04d.vtk", iteration);
	printf("# VTK: writing file %s\n", name);
	if (lbm_vtk_write_file(ld, kd, cd, iteration, name) != 0) {
		printf("ERROR: writing file %s failed.\n", name);
		return -1;
	}
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Seeded sphere packings (no counterpart in the reference, whose geometries
 * are box, channel, pipe, blocks and fluid only).
 *
 * Random numbers: splitmix64 expands the seed into the state and stream of a
 * PCG32 generator (O'Neill's pcg32 "XSH RR"); a uniform double takes two
 * draws (53 bits).
 *
 * Packing: random sequential addition of non-overlapping spheres (centres
 * uniform in the periodic box, radii uniform in [rmin, rmax]) until the target
 * voxel porosity is reached or `rsaAttempts` placements have been tried in a
 * row without success; if the packing has jammed above the target, spheres are
 * then added without the overlap test until the target is reached. A voxel
 * (x, y, z) is solid when its minimum-image distance to a centre is below the
 * radius. Random insertion of non-overlapping spheres jams near porosity 0.65
 * for radii 6..12, so lower targets need the second phase; the stats report
 * how many spheres it added. */

typedef struct { uint64_t state, inc; } lbmh_pcg32;

static uint64_t lbmh_splitmix64(uint64_t *x)
{
	uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
	return z ^ (z >> 31);
}

static uint32_t lbmh_pcg32_next(lbmh_pcg32 *r)
{
	uint64_t old = r->state;
	r->state = old * 6364136223846793005ull + r->inc;
	uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
	uint32_t rot = (uint32_t)(old >> 59);
	return (xs >> rot) | (xs << ((32 - rot) & 31));
}

static void lbmh_pcg32_seed(lbmh_pcg32 *r, uint64_t seed)
{
	uint64_t s = seed;
	r->state = lbmh_splitmix64(&s);
	r->inc = lbmh_splitmix64(&s) | 1ull;
	lbmh_pcg32_next(r);
}

static double lbmh_uniform(lbmh_pcg32 *r)
{
	uint64_t a = lbmh_pcg32_next(r) >> 5, b = lbmh_pcg32_next(r) >> 6;
	return (double)(a * 67108864ull + b) / 9007199254740992.0;
}

static double lbmh_pdist(double a, double b, int n)
{
	double d = fabs(a - b);
	return d > 0.5 * n ? n - d : d;
}

/* marks the voxels of one sphere solid; returns how many turned solid */
static long lbmh_voxelize(LatticeT *lat, const int dims[3], const double c[3], double r)
{
	long added = 0;
	const double r2 = r * r;
	const int lo[3] = { (int)floor(c[0] - r) - 1, (int)floor(c[1] - r) - 1, (int)floor(c[2] - r) - 1 };
	const int hi[3] = { (int)ceil(c[0] + r) + 1, (int)ceil(c[1] + r) + 1, (int)ceil(c[2] + r) + 1 };
	for (int z = lo[2]; z <= hi[2]; ++z) {
		const double dz = z - c[2];
		const int zz = ((z % dims[2]) + dims[2]) % dims[2];
		for (int y = lo[1]; y <= hi[1]; ++y) {
			const double dy = y - c[1];
			const int yy = ((y % dims[1]) + dims[1]) % dims[1];
			for (int x = lo[0]; x <= hi[0]; ++x) {
				const double dx = x - c[0];
				if (dx * dx + dy * dy + dz * dz >= r2) continue;
				const int xx = ((x % dims[0]) + dims[0]) % dims[0];
				LatticeT *v = &lat[lbmh_lidx(dims, xx, yy, zz)];
				if (*v != LAT_CELL_OBSTACLE) { *v = LAT_CELL_OBSTACLE; ++added; }
			}
		}
	}
	return added;
}

typedef struct { double c[3], r; } lbmh_sphere;

int lbm_geo_spheres(const int dims[3], uint64_t seed, double porosity, double rmin, double rmax,
                    int rsaAttempts, LatticeDesc *ld, double *stats)
{
	const int nx = dims[0], ny = dims[1], nz = dims[2];
	const long n = (long)nx * ny * nz;
	if (!(porosity > 0.0 && porosity <= 1.0) || !(rmin > 0.0) || rmax < rmin || n <= 0) {
		printf("ERROR: sphere packing needs 0 < porosity <= 1 and 0 < rmin <= rmax.\n");
		return -1;
	}
	LatticeT *lat = (LatticeT *)malloc(sizeof(LatticeT) * (size_t)n);
	if (!lat) { printf("ERROR: allocating the lattice mask failed.\n"); return -1; }
	for (long i = 0; i < n; ++i) lat[i] = LAT_CELL_FLUID;

	lbmh_pcg32 rng;
	lbmh_pcg32_seed(&rng, seed);

	/* bucket grid for the overlap test: bucket edge >= 2 rmax */
	int nb[3];
	for (int a = 0; a < 3; ++a) { nb[a] = (int)(dims[a] / (2.0 * rmax)); if (nb[a] < 1) nb[a] = 1; }
	const int nbt = nb[0] * nb[1] * nb[2];
	const int scanAll = nb[0] < 3 || nb[1] < 3 || nb[2] < 3;
	int *head = (int *)malloc(sizeof(int) * (size_t)nbt);
	for (int i = 0; i < nbt; ++i) head[i] = -1;
	int cap = 1024, ns = 0;
	lbmh_sphere *sp = (lbmh_sphere *)malloc(sizeof(lbmh_sphere) * (size_t)cap);
	int *next = (int *)malloc(sizeof(int) * (size_t)cap);

	const long target = (long)floor(porosity * (double)n);
	long fluid = n;
	long placedRsa = 0, placedOverlap = 0, fails = 0;
	double jamPorosity = -1.0;

	while (fluid > target) {
		lbmh_sphere s;
		s.c[0] = lbmh_uniform(&rng) * nx;
		s.c[1] = lbmh_uniform(&rng) * ny;
		s.c[2] = lbmh_uniform(&rng) * nz;
		s.r = rmin + (rmax - rmin) * lbmh_uniform(&rng);
		const int rsa = fails < rsaAttempts;
		if (!rsa && jamPorosity < 0.0) jamPorosity = (double)fluid / (double)n;

		int bc[3];
		for (int a = 0; a < 3; ++a) { bc[a] = (int)(s.c[a] / dims[a] * nb[a]); if (bc[a] >= nb[a]) bc[a] = nb[a] - 1; }
		if (rsa) {
			int overlap = 0;
			if (scanAll) {
				for (int i = 0; i < ns && !overlap; ++i) {
					const double dx = lbmh_pdist(s.c[0], sp[i].c[0], nx), dy = lbmh_pdist(s.c[1], sp[i].c[1], ny),
					             dz = lbmh_pdist(s.c[2], sp[i].c[2], nz);
					overlap = dx * dx + dy * dy + dz * dz < (s.r + sp[i].r) * (s.r + sp[i].r);
				}
			} else {
				for (int oz = -1; oz <= 1 && !overlap; ++oz)
				for (int oy = -1; oy <= 1 && !overlap; ++oy)
				for (int ox = -1; ox <= 1 && !overlap; ++ox) {
					const int b = (((bc[2] + oz + nb[2]) % nb[2]) * nb[1] + (bc[1] + oy + nb[1]) % nb[1]) * nb[0]
					              + (bc[0] + ox + nb[0]) % nb[0];
					for (int i = head[b]; i >= 0 && !overlap; i = next[i]) {
						const double dx = lbmh_pdist(s.c[0], sp[i].c[0], nx), dy = lbmh_pdist(s.c[1], sp[i].c[1], ny),
						             dz = lbmh_pdist(s.c[2], sp[i].c[2], nz);
						overlap = dx * dx + dy * dy + dz * dz < (s.r + sp[i].r) * (s.r + sp[i].r);
					}
				}
			}
			if (overlap) { ++fails; continue; }
			fails = 0;
			++placedRsa;
		} else {
			++placedOverlap;
		}
		if (ns == cap) {
			cap *= 2;
			sp = (lbmh_sphere *)realloc(sp, sizeof(lbmh_sphere) * (size_t)cap);
			next = (int *)realloc(next, sizeof(int) * (size_t)cap);
		}
		const int b = (bc[2] * nb[1] + bc[1]) * nb[0] + bc[0];
		sp[ns] = s;
		next[ns] = head[b];
		head[b] = ns;
		++ns;
		fluid -= lbmh_voxelize(lat, dims, s.c, s.r);
	}

	ld->Dims[0] = nx; ld->Dims[1] = ny; ld->Dims[2] = nz;
	ld->Lattice = lat;
	ld->nCells = (int)n;
	ld->nFluid = (int)fluid;
	ld->nObst = (int)(n - fluid);
	ld->nInlet = ld->nOutlet = 0;
	ld->PeriodicX = ld->PeriodicY = ld->PeriodicZ = 1;
	ld->Name = "spheres";
	if (stats) {
		stats[0] = (double)fluid / (double)n;
		stats[1] = (double)placedRsa;
		stats[2] = (double)placedOverlap;
		stats[3] = jamPorosity;
	}
	free(sp); free(next); free(head);
	return 0;
}

/* ------------------------------------------------------------------------ */
/* IEEE 754 binary16 conversions for the FP16 mirror (round to nearest even),
 * written from the format definition: 1 sign bit, 5 exponent bits (bias 15),
 * 10 fraction bits; subnormals below 2^-14. */

float lbmh_f16_to_f32(uint16_t h)
{
	const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
	const uint32_t ex = (h >> 10) & 0x1fu, fr = h & 0x3ffu;
	uint32_t bits;
	if (ex == 0) {
		if (fr == 0) bits = sign;
		else {
			/* subnormal: value = fr * 2^-24 */
			float v = (float)fr * 5.9604644775390625e-08f;
			memcpy(&bits, &v, 4);
			bits |= sign;
		}
	}
	else if (ex == 31) bits = sign | 0x7f800000u | (fr << 13);
	else bits = sign | ((ex + 112u) << 23) | (fr << 13);
	float out;
	memcpy(&out, &bits, 4);
	return out;
}

uint16_t lbmh_f32_to_f16(float f)
{
	uint32_t x;
	memcpy(&x, &f, 4);
	const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
	const uint32_t ax = x & 0x7fffffffu;
	if (ax >= 0x7f800000u) return sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u); /* NaN / inf */
	if (ax >= 0x477ff000u) return sign | 0x7c00u;                               /* rounds above 65504 */
	if (ax < 0x38800000u) {
		/* result subnormal or zero: round fr * 2^-24 to an integer, ties to even */
		float v;
		memcpy(&v, &ax, 4);
		float q = v * 16777216.0f; /* exact scaling by 2^24 */
		uint32_t i = (uint32_t)q;
		float rem = q - (float)i;
		if (rem > 0.5f || (rem == 0.5f && (i & 1u))) ++i;
		return sign | (uint16_t)i;
	}
	/* normal: drop 13 fraction bits with round to nearest even */
	uint32_t m = ax + 0xc8000000u; /* rebias exponent 127 -> 15 (subtract 112 << 23) */
	uint32_t r = m >> 13;
	uint32_t rest = m & 0x1fffu;
	if (rest > 0x1000u || (rest == 0x1000u && (r & 1u))) ++r;
	return sign | (uint16_t)r;
}
