/* lbm_oracle.c -- TEST INFRASTRUCTURE ONLY (see lbm_oracle.h).
 *
 * A plain-C restatement of the reference's D3Q19 TRT path, written to be read
 * beside the reference sources it follows (paths relative to the reference
 * project):
 *   geometry            src/Geometry.c:90-281
 *   padding             src/Padding.c:19-58,195-244
 *   AA full array       src/BenchKernelD3Q19AaCommon.c:309-637 (layout, fix-up
 *                       lists), src/BenchKernelD3Q19Aa.c:40-548 (steps)
 *   list AA (PV)        src/BenchKernelD3Q19ListAaPvCommon.c:471-823 (layout),
 *                       src/BenchKernelD3Q19ListAaPv.c:45-851 (steps, scalar
 *                       path arithmetic)
 *   list pull-split     src/BenchKernelD3Q19ListPullSplitNtCommon.c:422-797,
 *                       src/BenchKernelD3Q19ListPullSplitNt1SScalar.h
 *   list push/pull      src/BenchKernelD3Q19ListCommon.c:330-600 (layout),
 *   (two grids)         src/BenchKernelD3Q19List.c:114-344 (steps)
 *   body force          src/Kernel.c:759-803
 *   -verify init/check  src/Kernel.c:258-438, 451-625
 * The TRT magic parameter is an argument here (the reference hard-codes 1/12,
 * e.g. src/BenchKernelD3Q19Aa.c:71).
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define Q 19
#define QM 18
#define DC 18 /* centre direction is the last one */

/* Direction order N,S,E,W,NE,SE,NW,SW,T,TN,TE,TW,TS,B,BS,BN,BW,BE,C
 * (src/Kernel.h:89-140). */
static const int CX[Q] = { 0, 0, 1,-1, 1, 1,-1,-1, 0, 0, 1,-1, 0, 0, 0, 0,-1, 1, 0 };
static const int CY[Q] = { 1,-1, 0, 0, 1,-1, 1,-1, 0, 1, 0, 0,-1, 0,-1, 1, 0, 0, 0 };
static const int CZ[Q] = { 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1,-1,-1,-1,-1,-1, 0 };
static const int INV[Q] = { 1, 0, 3, 2, 7, 6, 5, 4,13,14,16,17,15, 8, 9,12,10,11,18 };
enum { N_=0, S_, E_, W_, NE_, SE_, NW_, SW_, T_, TN_, TE_, TW_, TS_, B_, BS_, BN_, BW_, BE_, C_ };

/* ------------------------------------------------------------------------ */
/* TRT collision, reference scalar operation order (src/BenchKernelD3Q19Aa.c:205-284).
 * out[i] is the post-collision value of direction i. */
typedef struct {
	double omegaEven, omegaOdd, w0, w1, w2, w1x3, w2x3, w1nh, w2nh;
} trt_t;

static trt_t trt_make(double omega, double lambda)
{
	trt_t t;
	t.omegaEven = omega;
	t.omegaOdd  = 1.0 / (0.5 + lambda / (1.0 / omega - 0.5));
	t.w0 = 1.0 / 3.0; t.w1 = 1.0 / 18.0; t.w2 = 1.0 / 36.0;
	t.w1x3 = t.w1 * 3.0; t.w1nh = t.w1 * 9.0 / 2.0;
	t.w2x3 = t.w2 * 3.0; t.w2nh = t.w2 * 9.0 / 2.0;
	return t;
}

static void trt_pair(const trt_t *t, const double *f, double *out, int a, int b, double ui,
                     double wnh, double wx3, double windep)
{
	double evenPart = t->omegaEven * (0.5 * (f[a] + f[b]) - ui * ui * wnh - windep);
	double oddPart  = t->omegaOdd  * (0.5 * (f[a] - f[b]) - ui * wx3);
	out[a] = f[a] - evenPart - oddPart;
	out[b] = f[b] - evenPart + oddPart;
}

static void trt_collide(const trt_t *t, const double *f, double *out)
{
	double ux = f[E_] + f[NE_] + f[SE_] + f[TE_] + f[BE_] -
	            f[W_] - f[NW_] - f[SW_] - f[TW_] - f[BW_];
	double uy = f[N_] + f[NE_] + f[NW_] + f[TN_] + f[BN_] -
	            f[S_] - f[SE_] - f[SW_] - f[TS_] - f[BS_];
	double uz = f[T_] + f[TE_] + f[TW_] + f[TN_] + f[TS_] -
	            f[B_] - f[BE_] - f[BW_] - f[BN_] - f[BS_];
	double dens = f[C_] +
	              f[N_]  + f[E_]  + f[S_]  + f[W_]  +
	              f[NE_] + f[SE_] + f[SW_] + f[NW_] +
	              f[T_]  + f[TN_] + f[TE_] + f[TS_] + f[TW_] +
	              f[B_]  + f[BN_] + f[BE_] + f[BS_] + f[BW_];
	double dit = dens - (ux * ux + uy * uy + uz * uz) * 3.0 / 2.0;

	out[C_] = f[C_] - t->omegaEven * (f[C_] - t->w0 * dit);

	double w1i = t->w1 * dit;
	trt_pair(t, f, out, N_, S_, uy, t->w1nh, t->w1x3, w1i);
	trt_pair(t, f, out, E_, W_, ux, t->w1nh, t->w1x3, w1i);
	trt_pair(t, f, out, T_, B_, uz, t->w1nh, t->w1x3, w1i);

	double w2i = t->w2 * dit;
	trt_pair(t, f, out, NW_, SE_, -ux + uy, t->w2nh, t->w2x3, w2i);
	trt_pair(t, f, out, NE_, SW_,  ux + uy, t->w2nh, t->w2x3, w2i);
	trt_pair(t, f, out, TW_, BE_, -ux + uz, t->w2nh, t->w2x3, w2i);
	trt_pair(t, f, out, TE_, BW_,  ux + uz, t->w2nh, t->w2x3, w2i);
	trt_pair(t, f, out, TS_, BN_, -uy + uz, t->w2nh, t->w2x3, w2i);
	trt_pair(t, f, out, TN_, BS_,  uy + uz, t->w2nh, t->w2x3, w2i);
}

/* Body-force increment of direction d, evaluated as src/Kernel.c:795. */
static double force_term(int d, double xforce)
{
	const double w0 = 1.0 / 3.0, w1 = 1.0 / 18.0, w2 = 1.0 / 36.0;
	const double w[Q] = { w1,w1,w1,w1,w2,w2,w2,w2,w1,w2,w2,w2,w2,w1,w2,w2,w2,w2,w0 };
	return 3.0 * w[d] * CX[d] * xforce;
}

/* ------------------------------------------------------------------------ */
/* Geometry (src/Geometry.c:90-281). */

#define LIDX(nx, ny, x, y, z) ((size_t)(z) * (nx) * (ny) + (size_t)(y) * (nx) + (x))

int orc_geometry(int type, int block_size, const int dims[3], const int periodic[3],
                 int *lat, int *info)
{
	int nx = dims[0], ny = dims[1], nz = dims[2];
	int p[3] = { periodic[0], periodic[1], periodic[2] };
	size_t n = (size_t)nx * ny * nz;

	for (size_t i = 0; i < n; ++i) lat[i] = 1;

	if (type == ORC_GEO_CHANNEL || type == ORC_GEO_BLOCKS || type == ORC_GEO_PIPE) p[0] = 1;
	else if (type == ORC_GEO_FLUID) { p[0] = 1; p[1] = 1; p[2] = 1; }

	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) {
		lat[LIDX(nx, ny, 0, y, z)]      = p[0] ? 1 : 0;
		lat[LIDX(nx, ny, nx - 1, y, z)] = p[0] ? 1 : 0;
	}
	for (int z = 0; z < nz; ++z) for (int x = 0; x < nx; ++x) {
		lat[LIDX(nx, ny, x, 0, z)]      = p[1] ? 1 : 0;
		lat[LIDX(nx, ny, x, ny - 1, z)] = p[1] ? 1 : 0;
	}
	for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
		lat[LIDX(nx, ny, x, y, 0)]      = p[2] ? 1 : 0;
		lat[LIDX(nx, ny, x, y, nz - 1)] = p[2] ? 1 : 0;
	}

	if (type == ORC_GEO_PIPE) {
		double cz = nz / 2.0 - 0.5, cy = ny / 2.0 - 0.5;
		double dmin = (ny < nz) ? ny : nz;
		double r = dmin / 2 - 1;
		double r2 = r * r;
		for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) {
			if ((z - cz) * (z - cz) + (y - cy) * (y - cy) >= r2)
				for (int x = 0; x < nx; ++x) lat[LIDX(nx, ny, x, y, z)] = 0;
		}
	}
	else if (type == ORC_GEO_BLOCKS && block_size > 0) {
		int b = block_size;
		for (int z = 0; z < nz; ++z) {
			if ((z % (2 * b)) < b) continue;
			for (int y = 0; y < ny; ++y) {
				if ((y % (2 * b)) < b) continue;
				for (int x = 0; x < nx; ++x)
					if ((x % (2 * b)) >= b) lat[LIDX(nx, ny, x, y, z)] = 0;
			}
		}
	}

	int nf = 0, no = 0;
	for (size_t i = 0; i < n; ++i) { if (lat[i] == 0) ++no; else ++nf; }
	info[0] = nf; info[1] = no; info[2] = 0; info[3] = 0;
	info[4] = periodic[0]; info[5] = periodic[1]; info[6] = periodic[2];
	info[7] = (p[0] ? 1 : 0) | (p[1] ? 2 : 0) | (p[2] ? 4 : 0);
	return 0;
}

/* ------------------------------------------------------------------------ */
/* SoA padding (src/Padding.c:19-58, 195-244). */

int orc_pad_cells(int n_cells, int pdf_bytes, int pad_mode, int n_pairs, const int *modulus, const int *offset)
{
	static const int auto_mod[2] = { 2 * 1024 * 1024 * 8, 256 * 64 };
	static const int auto_off[2] = { 2 * 1024 * 1024 + 512, 128 };
	const int *m = auto_mod, *o = auto_off;
	int k = 2;
	if (pad_mode == 1) k = 0;
	else if (pad_mode == 2) { m = modulus; o = offset; k = n_pairs; }

	for (int i = 0; i < k; ++i) {
		int pad;
		if (m[i] == 0) {
			pad = o[i] * pdf_bytes; /* as written in the reference (Padding.c:223) */
		} else {
			int mod_cells = m[i] / pdf_bytes;
			if (mod_cells == 0) return -1;
			int off_cells = o[i] / pdf_bytes;
			int rem = n_cells % mod_cells;
			pad = (off_cells + mod_cells - rem) % mod_cells;
		}
		n_cells += pad;
	}
	return n_cells;
}

/* ------------------------------------------------------------------------ */
/* List numbering and adjacency (src/BenchKernelD3Q19ListAaPvCommon.c:587-792,
 * src/BenchKernelD3Q19ListPullSplitNtCommon.c:488-755). */

typedef struct {
	int nx, ny, nz, nFluid, nCells;
	uint32_t *grid, *coords, *adj;
} orc_list_t;

/* pull: 1 pull adjacency with the pull-split cache-line pad, 2 pull adjacency
 * without it (two-grid list-pull-soa), 0 push adjacency. */
static int list_build(orc_list_t *L, int pull, const int dims[3], const int periodic[3], const int *lat,
                      const int blk_in[3], int pad_mode, int n_pairs, const int *modulus, const int *offset)
{
	int nx = dims[0], ny = dims[1], nz = dims[2];
	size_t n = (size_t)nx * ny * nz;
	int nf = 0;
	for (size_t i = 0; i < n; ++i) if (lat[i] != 0) ++nf;

	int nCells = orc_pad_cells(nf, 8, pad_mode, n_pairs, modulus, offset);
	if (nCells < 0) return -1;
	if (pull == 1) nCells = nCells + (8 - nCells % 8);

	L->nx = nx; L->ny = ny; L->nz = nz; L->nFluid = nf; L->nCells = nCells;
	L->grid = (uint32_t *)malloc(n * sizeof(uint32_t));
	L->coords = (uint32_t *)malloc((size_t)nf * 3 * sizeof(uint32_t) + 4);
	L->adj = (uint32_t *)malloc((size_t)nf * QM * sizeof(uint32_t) + 4);
	for (size_t i = 0; i < n; ++i) L->grid[i] = 0xffffffffu;

	int blk[3] = { blk_in ? blk_in[0] : 0, blk_in ? blk_in[1] : 0, blk_in ? blk_in[2] : 0 };
	if (blk[0] == 0) blk[0] = nx;
	if (blk[1] == 0) blk[1] = ny;
	if (blk[2] == 0) blk[2] = nz;

	uint32_t cnt = 0;
	for (int bx = 0; bx < nx; bx += blk[0])
	for (int by = 0; by < ny; by += blk[1])
	for (int bz = 0; bz < nz; bz += blk[2]) {
		int ex = bx + blk[0] < nx ? bx + blk[0] : nx;
		int ey = by + blk[1] < ny ? by + blk[1] : ny;
		int ez = bz + blk[2] < nz ? bz + blk[2] : nz;
		for (int x = bx; x < ex; ++x)
		for (int y = by; y < ey; ++y)
		for (int z = bz; z < ez; ++z) {
			size_t li = LIDX(nx, ny, x, y, z);
			if (lat[li] == 0) continue;
			L->grid[li] = cnt;
			L->coords[3 * (size_t)cnt + 0] = x;
			L->coords[3 * (size_t)cnt + 1] = y;
			L->coords[3 * (size_t)cnt + 2] = z;
			++cnt;
		}
	}

	int sgn = pull ? -1 : 1;
	for (int i = 0; i < nf; ++i) {
		int x = L->coords[3 * (size_t)i], y = L->coords[3 * (size_t)i + 1], z = L->coords[3 * (size_t)i + 2];
		for (int d = 0; d < QM; ++d) {
			int qx = x + sgn * CX[d], qy = y + sgn * CY[d], qz = z + sgn * CZ[d];
			int outx = qx < 0 || qx >= nx, outy = qy < 0 || qy >= ny, outz = qz < 0 || qz >= nz;
			uint32_t dst;
			if ((outx && periodic[0]) || (outy && periodic[1]) || (outz && periodic[2])) {
				/* every out-of-range coordinate wraps once one periodic axis is crossed */
				int px = qx < 0 ? nx - 1 : (qx >= nx ? 0 : qx);
				int py = qy < 0 ? ny - 1 : (qy >= ny ? 0 : qy);
				int pz = qz < 0 ? nz - 1 : (qz >= nz ? 0 : qz);
				size_t li = LIDX(nx, ny, px, py, pz);
				if (lat[li] == 0) dst = (uint32_t)INV[d] * nCells + i;
				else dst = (uint32_t)d * nCells + L->grid[li];
			}
			else if (outx || outy || outz) {
				dst = (uint32_t)INV[d] * nCells + i;
			}
			else {
				size_t li = LIDX(nx, ny, qx, qy, qz);
				if (lat[li] == 0) dst = (uint32_t)INV[d] * nCells + i;
				else dst = (uint32_t)d * nCells + L->grid[li];
			}
			L->adj[(size_t)i * QM + d] = dst;
		}
	}
	return 0;
}

static void list_free(orc_list_t *L)
{
	free(L->grid); free(L->coords); free(L->adj);
}

int orc_list_layout(int pull, const int dims[3], const int periodic[3], const int *lattice,
                    const int blk[3], int pad_mode, int n_pairs, const int *modulus, const int *offset,
                    uint32_t *grid_out, uint32_t *adj_out, int *counts_out)
{
	orc_list_t L;
	if (list_build(&L, pull, dims, periodic, lattice, blk, pad_mode, n_pairs, modulus, offset)) return -1;
	size_t n = (size_t)dims[0] * dims[1] * dims[2];
	if (grid_out) memcpy(grid_out, L.grid, n * sizeof(uint32_t));
	if (adj_out) memcpy(adj_out, L.adj, (size_t)L.nFluid * QM * sizeof(uint32_t));
	counts_out[0] = L.nFluid; counts_out[1] = L.nCells;
	list_free(&L);
	return 0;
}

/* ------------------------------------------------------------------------ */
/* A kernel state with the reference's logical node view (GetNode/SetNode). */

typedef struct {
	int kind;
	int nx, ny, nz;
	int iteration;
	/* AA full array */
	int gx, gy, gz;
	double *f;
	int *bbSrc, *bbDst, nBB;
	/* lists */
	orc_list_t L;
	double *g; /* second grid of the pull kernel */
} orc_state_t;

static size_t aa_i(const orc_state_t *s, int x, int y, int z, int d)
{ /* x,y,z in ghost coordinates; src/BenchKernelD3Q19AaCommon.h:80 */
	return (size_t)d * s->gx * s->gy * s->gz + (size_t)x * s->gy * s->gz + (size_t)y * s->gz + z;
}

/* AA logical view: src/BenchKernelD3Q19AaCommon.c:127-215.
 * List AA view: src/BenchKernelD3Q19ListAaPvCommon.c:127-223.
 * Pull view: src/BenchKernelD3Q19ListPullSplitNtCommon.c:118-182. */
static double *node_slot(orc_state_t *s, int x, int y, int z, int d)
{
	/* two-grid full array: push stores node x's PDFs at x, pull at x - c_d
	 * (src/BenchKernelD3Q19Common.c:120-196) */
	if (s->kind == ORC_KERNEL_PUSH_FA)
		return &s->f[aa_i(s, x + 1, y + 1, z + 1, d)];
	if (s->kind == ORC_KERNEL_PULL_FA)
		return &s->f[aa_i(s, x + 1 - CX[d], y + 1 - CY[d], z + 1 - CZ[d], d)];
	if (s->kind == ORC_KERNEL_AA) {
		if (s->iteration % 2 == 0)
			return &s->f[aa_i(s, x + 1 - CX[d], y + 1 - CY[d], z + 1 - CZ[d], INV[d])];
		return &s->f[aa_i(s, x + 1, y + 1, z + 1, d)];
	}
	uint32_t node = s->L.grid[LIDX(s->nx, s->ny, x, y, z)];
	if (s->kind == ORC_KERNEL_LIST_AA && s->iteration % 2 == 0 && d != DC)
		return &s->f[s->L.adj[(size_t)node * QM + INV[d]]];
	return &s->f[(size_t)d * s->L.nCells + node];
}

static void get_node(orc_state_t *s, int x, int y, int z, double *p)
{
	for (int d = 0; d < Q; ++d) p[d] = *node_slot(s, x, y, z, d);
}

static void set_node(orc_state_t *s, int x, int y, int z, const double *p)
{
	for (int d = 0; d < Q; ++d) *node_slot(s, x, y, z, d) = p[d];
}

static void add_body_force(orc_state_t *s, const int *lat, double xforce)
{
	double ft[Q];
	for (int d = 0; d < Q; ++d) ft[d] = force_term(d, xforce);
	#pragma omp parallel for collapse(2)
	for (int z = 0; z < s->nz; ++z) for (int y = 0; y < s->ny; ++y) {
		for (int x = 0; x < s->nx; ++x) {
			if (lat[LIDX(s->nx, s->ny, x, y, z)] == 0) continue;
			for (int d = 0; d < Q; ++d) {
				double *slot = node_slot(s, x, y, z, d);
				*slot = *slot + ft[d];
			}
		}
	}
}

/* KernelSetInitialDensity / KernelSetInitialVelocity (src/Kernel.c:258-438):
 * f_i = 3 w_i omega (rho/3 - u^2/2 + ...), with the density ramp rho_in ->
 * rho_out along x for the first and rho = 1 for the second. */
static void equilibrium_like_reference(double omega, double dens, double ux, double uy, double uz, double *p)
{
	const double w0 = 1.0 / 3.0, w1 = 1.0 / 18.0, w2 = 1.0 / 36.0;
	double ow0 = 3.0 * w0 * omega, ow1 = 3.0 * w1 * omega, ow2 = 3.0 * w2 * omega;
	double third = 1.0 / 3.0;
	double dit = third * dens - 0.5 * (ux * ux + uy * uy + uz * uz);
#define SQ(a) ((a) * (a))
	p[C_]  = ow0 * (dit);
	p[NW_] = ow2 * (dit - (ux - uy) + 1.5 * SQ(ux - uy));
	p[SE_] = ow2 * (dit + (ux - uy) + 1.5 * SQ(ux - uy));
	p[NE_] = ow2 * (dit + (ux + uy) + 1.5 * SQ(ux + uy));
	p[SW_] = ow2 * (dit - (ux + uy) + 1.5 * SQ(ux + uy));
	p[TW_] = ow2 * (dit - (ux - uz) + 1.5 * SQ(ux - uz));
	p[BE_] = ow2 * (dit + (ux - uz) + 1.5 * SQ(ux - uz));
	p[TE_] = ow2 * (dit + (ux + uz) + 1.5 * SQ(ux + uz));
	p[BW_] = ow2 * (dit - (ux + uz) + 1.5 * SQ(ux + uz));
	p[TS_] = ow2 * (dit - (uy - uz) + 1.5 * SQ(uy - uz));
	p[BN_] = ow2 * (dit + (uy - uz) + 1.5 * SQ(uy - uz));
	p[TN_] = ow2 * (dit + (uy + uz) + 1.5 * SQ(uy + uz));
	p[BS_] = ow2 * (dit - (uy + uz) + 1.5 * SQ(uy + uz));
	p[N_]  = ow1 * (dit + uy + 1.5 * SQ(uy));
	p[S_]  = ow1 * (dit - uy + 1.5 * SQ(uy));
	p[E_]  = ow1 * (dit + ux + 1.5 * SQ(ux));
	p[W_]  = ow1 * (dit - ux + 1.5 * SQ(ux));
	p[T_]  = ow1 * (dit + uz + 1.5 * SQ(uz));
	p[B_]  = ow1 * (dit - uz + 1.5 * SQ(uz));
#undef SQ
}

static void init_verify(orc_state_t *s, const int *lat, double omega, double rho_in, double rho_out)
{
	int nx = s->nx, ny = s->ny, nz = s->nz;
	double p[Q];
	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
		if (lat[LIDX(nx, ny, x, y, z)] == 0) continue;
		double dens = rho_in + (rho_out - rho_in) * (x) / (nx - 1.0);
		equilibrium_like_reference(omega, dens, 0.0, 0.0, 0.0, p);
		set_node(s, x, y, z, p);
	}
	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
		if (lat[LIDX(nx, ny, x, y, z)] != 1) continue;
		equilibrium_like_reference(omega, 1.0, 0.0, 0.0, 0.0, p);
		set_node(s, x, y, z, p);
	}
}

/* ------------------------------------------------------------------------ */
/* AA full array: ghost-padded (n+2)^3 SoA, z fastest; fix-up lists for
 * periodic and bounce-back PDFs (src/BenchKernelD3Q19AaCommon.c:446-621). */

/* Fix-up lists of the two-grid full-array pull kernel
 * (src/BenchKernelD3Q19Common.c:531-660, PROP_MODEL_PULL): the neighbour a
 * node pulls from is x - c_d; a wall or a wall behind a periodic wrap gets
 * the node's own inverse PDF, a periodic ghost the image's PDF. */
static void fa_build_pull_fixup(orc_state_t *s, const int *lat, const int periodic[3])
{
	int lx = s->nx, ly = s->ny, lz = s->nz;
	int cap = 0;
	for (size_t i = 0; i < (size_t)lx * ly * lz; ++i) if (lat[i] != 0) cap += Q;
	s->bbSrc = (int *)malloc(sizeof(int) * (size_t)(cap + 1));
	s->bbDst = (int *)malloc(sizeof(int) * (size_t)(cap + 1));
	int k = 0;
	for (int x = 0; x < lx; ++x) for (int y = 0; y < ly; ++y) for (int z = 0; z < lz; ++z) {
		if (lat[LIDX(lx, ly, x, y, z)] == 0) continue;
		for (int d = 0; d < Q; ++d) {
			int nx = x - CX[d], ny = y - CY[d], nz = z - CZ[d];
			int ox = nx < 0 || nx >= lx, oy = ny < 0 || ny >= ly, oz = nz < 0 || nz >= lz;
			if ((ox && periodic[0]) || (oy && periodic[1]) || (oz && periodic[2])) {
				int px = nx < 0 ? lx - 1 : (nx >= lx ? 0 : nx);
				int py = ny < 0 ? ly - 1 : (ny >= ly ? 0 : ny);
				int pz = nz < 0 ? lz - 1 : (nz >= lz ? 0 : nz);
				if (lat[LIDX(lx, ly, px, py, pz)] == 0)
					s->bbSrc[k] = (int)aa_i(s, x + 1, y + 1, z + 1, INV[d]);
				else
					s->bbSrc[k] = (int)aa_i(s, px + 1, py + 1, pz + 1, d);
				s->bbDst[k] = (int)aa_i(s, nx + 1, ny + 1, nz + 1, d);
				++k;
			}
			else if (ox || oy || oz) {
				continue;
			}
			else if (lat[LIDX(lx, ly, nx, ny, nz)] == 0) {
				s->bbSrc[k] = (int)aa_i(s, x + 1, y + 1, z + 1, INV[d]);
				s->bbDst[k] = (int)aa_i(s, nx + 1, ny + 1, nz + 1, d);
				++k;
			}
		}
	}
	s->nBB = k;
}

static void aa_build_fixup(orc_state_t *s, const int *lat, const int periodic[3])
{
	int lx = s->nx, ly = s->ny, lz = s->nz;
	int cap = 0;
	for (size_t i = 0; i < (size_t)lx * ly * lz; ++i) if (lat[i] != 0) cap += Q;
	s->bbSrc = (int *)malloc(sizeof(int) * (size_t)(cap + 1));
	s->bbDst = (int *)malloc(sizeof(int) * (size_t)(cap + 1));
	int k = 0;
	for (int x = 0; x < lx; ++x) for (int y = 0; y < ly; ++y) for (int z = 0; z < lz; ++z) {
		if (lat[LIDX(lx, ly, x, y, z)] == 0) continue;
		for (int d = 0; d < Q; ++d) {
			int nx = x + CX[d], ny = y + CY[d], nz = z + CZ[d];
			int ox = nx < 0 || nx >= lx, oy = ny < 0 || ny >= ly, oz = nz < 0 || nz >= lz;
			if ((ox && periodic[0]) || (oy && periodic[1]) || (oz && periodic[2])) {
				int px = nx < 0 ? lx - 1 : (nx >= lx ? 0 : nx);
				int py = ny < 0 ? ly - 1 : (ny >= ly ? 0 : ny);
				int pz = nz < 0 ? lz - 1 : (nz >= lz ? 0 : nz);
				s->bbSrc[k] = (int)aa_i(s, nx + 1, ny + 1, nz + 1, d);
				if (lat[LIDX(lx, ly, px, py, pz)] == 0)
					s->bbDst[k] = (int)aa_i(s, x + 1, y + 1, z + 1, INV[d]);
				else
					s->bbDst[k] = (int)aa_i(s, px + 1, py + 1, pz + 1, d);
				++k;
			}
			else if (ox || oy || oz) {
				continue;
			}
			else if (lat[LIDX(lx, ly, nx, ny, nz)] == 0) {
				s->bbSrc[k] = (int)aa_i(s, nx + 1, ny + 1, nz + 1, d);
				s->bbDst[k] = (int)aa_i(s, x + 1, y + 1, z + 1, INV[d]);
				++k;
			}
		}
	}
	s->nBB = k;
}

static void aa_even(orc_state_t *s, const int *lat, const trt_t *t)
{
	#pragma omp parallel for collapse(2)
	for (int x = 0; x < s->nx; ++x) for (int y = 0; y < s->ny; ++y) {
		for (int z = 0; z < s->nz; ++z) {
			if (lat[LIDX(s->nx, s->ny, x, y, z)] == 0) continue;
			double f[Q], o[Q];
			for (int d = 0; d < Q; ++d) f[d] = s->f[aa_i(s, x + 1, y + 1, z + 1, d)];
			trt_collide(t, f, o);
			for (int d = 0; d < Q; ++d) s->f[aa_i(s, x + 1, y + 1, z + 1, INV[d])] = o[d];
		}
	}
}

static void aa_odd(orc_state_t *s, const trt_t *t)
{
	/* every interior cell, obstacles included (src/BenchKernelD3Q19Aa.c:380-491) */
	#pragma omp parallel for collapse(2)
	for (int x = 0; x < s->nx; ++x) for (int y = 0; y < s->ny; ++y) {
		for (int z = 0; z < s->nz; ++z) {
			int gx = x + 1, gy = y + 1, gz = z + 1;
			double f[Q], o[Q];
			for (int d = 0; d < Q; ++d) f[d] = s->f[aa_i(s, gx - CX[d], gy - CY[d], gz - CZ[d], INV[d])];
			trt_collide(t, f, o);
			for (int d = 0; d < Q; ++d) s->f[aa_i(s, gx + CX[d], gy + CY[d], gz + CZ[d], d)] = o[d];
		}
	}
}

/* Two-grid full array (src/BenchKernelD3Q19.c:114-334): every interior cell,
 * obstacles included, from grid f into grid g -- push: own PDFs in, PDF d out
 * to x + c_d; pull: PDF d in from x - c_d, own PDFs out. The fix-up lists
 * then run on g. */
static void fa_step(orc_state_t *s, const trt_t *t, int pull)
{
	#pragma omp parallel for collapse(2)
	for (int x = 0; x < s->nx; ++x) for (int y = 0; y < s->ny; ++y) {
		for (int z = 0; z < s->nz; ++z) {
			int gx = x + 1, gy = y + 1, gz = z + 1;
			double f[Q], o[Q];
			for (int d = 0; d < Q; ++d)
				f[d] = pull ? s->f[aa_i(s, gx - CX[d], gy - CY[d], gz - CZ[d], d)] : s->f[aa_i(s, gx, gy, gz, d)];
			trt_collide(t, f, o);
			for (int d = 0; d < Q; ++d) {
				if (pull) s->g[aa_i(s, gx, gy, gz, d)] = o[d];
				else s->g[aa_i(s, gx + CX[d], gy + CY[d], gz + CZ[d], d)] = o[d];
			}
		}
	}
	for (int i = 0; i < s->nBB; ++i) s->g[s->bbDst[i]] = s->g[s->bbSrc[i]];
}

/* ------------------------------------------------------------------------ */
/* List AA (src/BenchKernelD3Q19ListAaPv.c:161-470 even, 472-851 odd). */

static void list_even(orc_state_t *s, const trt_t *t)
{
	size_t nc = (size_t)s->L.nCells;
	#pragma omp parallel for
	for (int n = 0; n < s->L.nFluid; ++n) {
		double f[Q], o[Q];
		for (int d = 0; d < Q; ++d) f[d] = s->f[d * nc + n];
		trt_collide(t, f, o);
		for (int d = 0; d < Q; ++d) s->f[INV[d] * nc + n] = o[d];
	}
}

static void list_odd(orc_state_t *s, const trt_t *t)
{
	size_t nc = (size_t)s->L.nCells;
	#pragma omp parallel for
	for (int n = 0; n < s->L.nFluid; ++n) {
		const uint32_t *a = s->L.adj + (size_t)n * QM;
		double f[Q], o[Q];
		for (int d = 0; d < QM; ++d) f[d] = s->f[a[INV[d]]];
		f[DC] = s->f[DC * nc + n];
		trt_collide(t, f, o);
		for (int d = 0; d < QM; ++d) s->f[a[d]] = o[d];
		s->f[DC * nc + n] = o[DC];
	}
}

/* One half of a list AA step pair on a caller-supplied layout (nodes
 * [0, n_nodes) of f[d * n_cells + node], push adjacency adj[node * 18 + d]),
 * for checking decomposed runs whose slabs hold ghost nodes past n_nodes.
 * The arithmetic is list_even / list_odd above. The reference's per-step body
 * force (src/Kernel.c:759-803, add_body_force) is added to each slot once, at
 * the access that follows it: the even step's force when the odd step loads a
 * value, the odd step's force when it stores one (a slot it bounces into
 * carries the force of the inverse direction). That is the same single
 * addition per slot as the separate pass, so every complete pair leaves the
 * bits orc_run leaves, and a slot that another slab updates between the two
 * halves receives its force from the node that reads it. */
int orc_list_aa_half(int odd, int n_nodes, int n_cells, const uint32_t *adj, double *f,
                     double omega, double lambda, double xforce)
{
	return orc_list_aa_half_range(odd, 0, n_nodes, n_cells, adj, f, omega, lambda, xforce);
}

/* The same over nodes [n0, n1) only (adj indexed by node: adj[n * 18]). */
int orc_list_aa_half_range(int odd, int n0, int n1, int n_cells, const uint32_t *adj, double *f,
                           double omega, double lambda, double xforce)
{
	const trt_t t = trt_make(omega, lambda);
	double ft[Q];
	for (int d = 0; d < Q; ++d) ft[d] = force_term(d, xforce);
	const size_t nc = (size_t)n_cells;
	for (int n = n0; n < n1; ++n) {
		double p[Q], o[Q];
		if (!odd) {
			for (int d = 0; d < Q; ++d) p[d] = f[d * nc + n];
			trt_collide(&t, p, o);
			for (int d = 0; d < Q; ++d) f[INV[d] * nc + n] = o[d];
			continue;
		}
		const uint32_t *a = adj + (size_t)n * QM;
		for (int d = 0; d < QM; ++d) p[d] = f[a[INV[d]]] + ft[d];
		p[DC] = f[DC * nc + n] + ft[DC];
		trt_collide(&t, p, o);
		for (int d = 0; d < QM; ++d) {
			const int bounce = a[d] == (uint32_t)(INV[d] * nc + n);
			f[a[d]] = o[d] + (bounce ? ft[INV[d]] : ft[d]);
		}
		f[DC * nc + n] = o[DC] + ft[DC];
	}
	return 0;
}

/* List pull (src/BenchKernelD3Q19ListPullSplitNt1SScalar.h): gather through the
 * pull adjacency from the source grid, write the destination grid. */
static void list_pull(orc_state_t *s, const trt_t *t)
{
	size_t nc = (size_t)s->L.nCells;
	#pragma omp parallel for
	for (int n = 0; n < s->L.nFluid; ++n) {
		const uint32_t *a = s->L.adj + (size_t)n * QM;
		double f[Q], o[Q];
		f[DC] = s->f[DC * nc + n];
		for (int d = 0; d < QM; ++d) f[d] = s->f[a[d]];
		trt_collide(t, f, o);
		for (int d = 0; d < Q; ++d) s->g[d * nc + n] = o[d];
	}
}

/* Two-grid list push (src/BenchKernelD3Q19List.c:114-320, PROP_MODEL_PUSH):
 * the node's own PDFs from the source grid, each post-collision PDF written
 * through the push adjacency into the destination grid. */
static void list_push2(orc_state_t *s, const trt_t *t)
{
	size_t nc = (size_t)s->L.nCells;
	#pragma omp parallel for
	for (int n = 0; n < s->L.nFluid; ++n) {
		const uint32_t *a = s->L.adj + (size_t)n * QM;
		double f[Q], o[Q];
		for (int d = 0; d < Q; ++d) f[d] = s->f[d * nc + n];
		trt_collide(t, f, o);
		for (int d = 0; d < QM; ++d) s->g[a[d]] = o[d];
		s->g[DC * nc + n] = o[DC];
	}
}

/* ------------------------------------------------------------------------ */

int orc_run(int kernel, const int dims[3], const int periodic[3], const int *lattice,
            double omega, double lambda, double xforce, double rho_in, double rho_out,
            int iterations, int init_mode, const double *init_pdfs, double *out_pdfs,
            const int blk[3], int pad_mode)
{
	orc_state_t s;
	memset(&s, 0, sizeof(s));
	s.kind = kernel;
	s.nx = dims[0]; s.ny = dims[1]; s.nz = dims[2];
	s.iteration = -1;
	size_t ncell = (size_t)s.nx * s.ny * s.nz;

	const int fa = kernel == ORC_KERNEL_PUSH_FA || kernel == ORC_KERNEL_PULL_FA;
	if (kernel == ORC_KERNEL_AA || fa) {
		s.gx = s.nx + 2; s.gy = s.ny + 2; s.gz = s.nz + 2;
		s.f = (double *)calloc((size_t)Q * s.gx * s.gy * s.gz, sizeof(double));
		if (kernel == ORC_KERNEL_PULL_FA)
			fa_build_pull_fixup(&s, lattice, periodic);
		else
			aa_build_fixup(&s, lattice, periodic); /* the push lists of the two-grid kernel are the same */
		if (fa) s.g = (double *)calloc((size_t)Q * s.gx * s.gy * s.gz, sizeof(double));
	} else {
		const int pull = kernel == ORC_KERNEL_LIST_PULL ? 1 : (kernel == ORC_KERNEL_LIST_PULL2 ? 2 : 0);
		if (list_build(&s.L, pull, dims, periodic, lattice, blk, pad_mode, 0, NULL, NULL))
			return -1;
		s.f = (double *)calloc((size_t)Q * s.L.nCells, sizeof(double));
		if (kernel != ORC_KERNEL_LIST_AA)
			s.g = (double *)calloc((size_t)Q * s.L.nCells, sizeof(double));
	}

	if (init_mode == ORC_INIT_VERIFY) {
		init_verify(&s, lattice, omega, rho_in, rho_out);
	} else if (init_mode == ORC_INIT_PDFS) {
		for (int z = 0; z < s.nz; ++z) for (int y = 0; y < s.ny; ++y) for (int x = 0; x < s.nx; ++x) {
			size_t c = LIDX(s.nx, s.ny, x, y, z);
			if (lattice[c] == 0) continue;
			set_node(&s, x, y, z, init_pdfs + c * Q);
		}
	}

	trt_t t = trt_make(omega, lambda);

	if (kernel == ORC_KERNEL_AA || kernel == ORC_KERNEL_LIST_AA) {
		/* both AA kernels advance in even/odd pairs */
		for (int it = 0; it < iterations; it += 2) {
			if (kernel == ORC_KERNEL_AA) {
				aa_even(&s, lattice, &t);
				for (int i = 0; i < s.nBB; ++i) s.f[s.bbSrc[i]] = s.f[s.bbDst[i]];
			} else {
				list_even(&s, &t);
			}
			s.iteration = it;
			add_body_force(&s, lattice, xforce);

			if (kernel == ORC_KERNEL_AA) {
				aa_odd(&s, &t);
				for (int i = 0; i < s.nBB; ++i) s.f[s.bbDst[i]] = s.f[s.bbSrc[i]];
			} else {
				list_odd(&s, &t);
			}
			s.iteration = it + 1;
			add_body_force(&s, lattice, xforce);
		}
	} else {
		for (int it = 0; it < iterations; ++it) {
			if (fa)
				fa_step(&s, &t, kernel == ORC_KERNEL_PULL_FA);
			else if (kernel == ORC_KERNEL_LIST_PUSH2)
				list_push2(&s, &t);
			else
				list_pull(&s, &t);
			double *tmp = s.f; s.f = s.g; s.g = tmp;
			add_body_force(&s, lattice, xforce);
		}
	}

	if (out_pdfs) {
		for (int z = 0; z < s.nz; ++z) for (int y = 0; y < s.ny; ++y) for (int x = 0; x < s.nx; ++x) {
			size_t c = LIDX(s.nx, s.ny, x, y, z);
			if (lattice[c] == 0) continue;
			get_node(&s, x, y, z, out_pdfs + c * Q);
		}
	}
	(void)ncell;

	free(s.f); free(s.g); free(s.bbSrc); free(s.bbDst);
	if (kernel != ORC_KERNEL_AA && !fa) list_free(&s.L);
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Poiseuille check (src/Kernel.c:451-625). */

double orc_verify_error(const int dims[3], const int *lat, const double *pdfs, double omega, double xforce)
{
	int nx = dims[0], ny = dims[1], nz = dims[2];
	double visc = (1.0 / omega - 0.5) / 3.0;
	double *slice = (double *)malloc(sizeof(double) * (size_t)ny * nz);
	int xp = nx / 2;
	for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) {
		size_t c = LIDX(nx, ny, xp, y, z);
		if (lat[c] != 0) {
			const double *p = pdfs + c * Q;
			double ux = p[E_] + p[NE_] + p[SE_] + p[TE_] + p[BE_] -
			            p[W_] - p[NW_] - p[SW_] - p[TW_] - p[BW_];
			ux += 0.5 * xforce;
			slice[y * nz + z] = ux;
		} else {
			slice[y * nz + z] = 0.0;
		}
	}
	int even = (ny % 2 == 0);
	int y = (ny - even - 1) / 2;
	double center = ny / 2.0;
	double dmin = (double)ny;
	double r2min = (dmin / 2.0 - 1.0) * (dmin / 2.0 - 1.0);
	double dev = 0.0;
	for (int z = 0; z < nz; ++z) {
		double r2 = (z - center + 0.5) * (z - center + 0.5);
		double ua = (r2 >= r2min) ? 0.0 : xforce * (r2min - r2) / (2.0 * visc);
		double us = even ? (slice[y * nz + z] + slice[(y + 1) * nz + z]) / 2.0 : slice[y * nz + z];
		if (ua != 0.0) {
			double rel = fabs(ua - us) / ua;
			dev += rel * rel;
		}
	}
	free(slice);
	return sqrt(dev);
}
