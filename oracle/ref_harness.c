// ref_harness.c -- TEST INFRASTRUCTURE ONLY (never shipped, never timed as the
// product). Links against the reference implementation's own objects, which
// oracle/Makefile compiles unmodified from the reference sources, and drives
// its kernels through the reference's own kernel table (KernelFunctions.h
// g_kernels[], src/KernelFunctions.h:56-188) exactly as src/Main.c does:
//
//   GeoCreateByStr / caller-supplied LatticeDesc   (src/Main.c:476)
//   kf->Init(&ld, &kd, &p)                          (src/Main.c:560)
//   KernelSetInitialDensity / ...Velocity           (src/Main.c:562-567)
//   kd->Kernel(&ld, kd, &cd)                        (src/Main.c:574)
//   kd->GetNode over all fluid nodes                (src/Kernel.c:209-254)
//   kf->Deinit(&ld, &kd)                            (src/Main.c:592)
//
// It exposes flat C entry points for the Python tests (ctypes).
#include "BenchKernelD3Q19ListAaCommon.h"
#include "KernelFunctions.h"
#include "Geometry.h"
#include "Pinning.h"

#include <malloc.h>
#include <stdint.h>
#include <strings.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static KernelFunctions *refh_find(const char *name)
{
	for (int j = 0; j < (int)(sizeof(g_kernels) / sizeof(g_kernels[0])); ++j) {
		if (!strcasecmp(name, g_kernels[j].Name)) return &g_kernels[j];
	}
	return NULL;
}

// Number of kernels in the reference's table, and the name of entry i.
int refh_kernel_count(void) { return (int)(sizeof(g_kernels) / sizeof(g_kernels[0])); }
const char *refh_kernel_name(int i) { return g_kernels[i].Name; }

int refh_set_threads(int n)
{
#ifdef _OPENMP
	if (n > 0) omp_set_num_threads(n);
	return omp_get_max_threads();
#else
	(void)n;
	return 1;
#endif
}

// Pins OpenMP thread i to the i-th CPU of cpuList ("0,2,4,..."), as the
// reference's -pin does (src/Main.c:505-530, PinCurrentThreadByCpuList of
// src/Pinning.c). Returns the number of threads whose pinning failed.
int refh_pin(const char *cpuList)
{
	int failed = 0;
#ifdef _OPENMP
	#pragma omp parallel reduction(+:failed)
	{
		if (PinCurrentThreadByCpuList(cpuList, omp_get_thread_num()) != 0) failed += 1;
	}
#else
	(void)cpuList;
#endif
	return failed;
}

// Builds a geometry with the reference's GeoCreateByStr (src/Geometry.c:37-88).
// lattice_out: nX*nY*nZ ints (x fastest). info_out[0..7]: nFluid, nObst,
// nInlet, nOutlet, ld.PeriodicX/Y/Z, and the periodic flags the geometry
// routine wrote back into the caller's array packed as bits (x=1,y=2,z=4).
int refh_geometry(const char *geo, const int dims[3], const int periodic[3], int *lattice_out, int *info_out)
{
	int d[3] = { dims[0], dims[1], dims[2] };
	int p[3] = { periodic[0], periodic[1], periodic[2] };
	LatticeDesc ld;
	GeoCreateByStr(geo, d, p, &ld);
	size_t n = (size_t)d[0] * d[1] * d[2];
	memcpy(lattice_out, ld.Lattice, n * sizeof(int));
	info_out[0] = ld.nFluid; info_out[1] = ld.nObst;
	info_out[2] = ld.nInlet; info_out[3] = ld.nOutlet;
	info_out[4] = ld.PeriodicX; info_out[5] = ld.PeriodicY; info_out[6] = ld.PeriodicZ;
	info_out[7] = (p[0] ? 1 : 0) | (p[1] ? 2 : 0) | (p[2] ? 4 : 0);
	free(ld.Lattice);
	return 0;
}

static void refh_fill_ld(LatticeDesc *ld, const int dims[3], const int periodic[3], int *lattice)
{
	ld->Dims[0] = dims[0]; ld->Dims[1] = dims[1]; ld->Dims[2] = dims[2];
	ld->Lattice = lattice;
	ld->nCells = dims[0] * dims[1] * dims[2];
	ld->PeriodicX = periodic[0]; ld->PeriodicY = periodic[1]; ld->PeriodicZ = periodic[2];
	ld->Name = "harness";
	ld->nFluid = ld->nObst = ld->nInlet = ld->nOutlet = 0;
	for (int i = 0; i < ld->nCells; ++i) {
		switch (lattice[i]) {
			case LAT_CELL_OBSTACLE: ld->nObst++; break;
			case LAT_CELL_INLET:    ld->nInlet++; ld->nFluid++; break;
			case LAT_CELL_OUTLET:   ld->nOutlet++; ld->nFluid++; break;
			default:                ld->nFluid++; break;
		}
	}
}

static int is_list_aa(const char *name)
{
	return !strncasecmp(name, "list-aa", 7);
}

// Runs `iterations` steps of reference kernel `name` on the given mask.
//   init_mode 0: the kernel's own initialisation (PDFs 0.0, as benchmark runs)
//   init_mode 1: KernelSetInitialDensity + KernelSetInitialVelocity (-verify)
//   init_mode 2: SetNode from init_pdfs (cells x fastest, 19 PDFs per cell)
// out_pdfs (optional): GetNode of every non-obstacle cell after the run,
// same layout; obstacle cells are left untouched.
// Returns the kernel's own Duration (seconds) through *duration.
int refh_run(const char *name, const int dims[3], const int periodic[3], int *lattice,
             double omega, double xforce, double rho_in, double rho_out, int iterations,
             int init_mode, const double *init_pdfs, double *out_pdfs,
             int n_kargs, char **kargs, double *duration)
{
	KernelFunctions *kf = refh_find(name);
	if (kf == NULL) return -1;

	// With a non-periodic face whose cells are fluid (e.g. -geometry channel
	// without -periodic-x), the AA kernels read ghost-layer PDFs that
	// D3Q19AaInit never writes (src/BenchKernelD3Q19AaCommon.c:376-443) on
	// the first odd step. In a fresh process those large arrays come from
	// fresh zero pages. glibc's M_PERTURB with 0xff fills every new block with
	// the complement of 0xff, i.e. zero bytes, which keeps that true for every
	// run inside one long-lived test process.
	mallopt(M_PERTURB, 0xff);

	LatticeDesc ld;
	refh_fill_ld(&ld, dims, periodic, lattice);

	CaseData cd;
	cd.MaxIterations = iterations;
	cd.RhoIn = rho_in; cd.RhoOut = rho_out;
	cd.Omega = omega;
	cd.Ux = cd.Uy = cd.Uz = 0.0;
	cd.VtkOutput = 0; cd.VtkModulus = 100; cd.StatisticsModulus = 100;
	cd.XForce = xforce;

	Parameters p;
	p.nArgs = 0; p.Args = NULL;
	p.nKernelArgs = n_kargs; p.KernelArgs = kargs;

	KernelData *kd = NULL;
	kf->Init(&ld, &kd, &p);

	// The list-AA kernels leave KernelDataList.Iteration uninitialised in
	// Init (src/BenchKernelD3Q19ListAaPvCommon.c:471-823); their first step is
	// an even (local) step, which reads the natural layout, so the harness
	// selects that layout for SetNode explicitly.
	if (is_list_aa(name)) ((KernelDataList *)kd)->Iteration = -1;

	int nX = dims[0], nY = dims[1], nZ = dims[2];

	if (init_mode == 1) {
		KernelSetInitialDensity(&ld, kd, &cd);
		KernelSetInitialVelocity(&ld, kd, &cd);
	}
	else if (init_mode == 2) {
		for (int z = 0; z < nZ; ++z) for (int y = 0; y < nY; ++y) for (int x = 0; x < nX; ++x) {
			size_t c = (size_t)z * nX * nY + (size_t)y * nX + x;
			if (lattice[c] == LAT_CELL_OBSTACLE) continue;
			double pdfs[N_D3Q19];
			memcpy(pdfs, init_pdfs + c * N_D3Q19, sizeof(pdfs));
			kd->SetNode(kd, x, y, z, pdfs);
		}
	}

	if (iterations > 0) kd->Kernel(&ld, kd, &cd);
	if (duration) *duration = kd->Duration;

	if (out_pdfs) {
		for (int z = 0; z < nZ; ++z) for (int y = 0; y < nY; ++y) for (int x = 0; x < nX; ++x) {
			size_t c = (size_t)z * nX * nY + (size_t)y * nX + x;
			if (lattice[c] == LAT_CELL_OBSTACLE) continue;
			kd->GetNode(kd, x, y, z, out_pdfs + c * N_D3Q19);
		}
	}

	kf->Deinit(&ld, &kd);
	return 0;
}

// Runs the reference Init of a list kernel and copies its numbering and
// adjacency out: grid_out (nX*nY*nZ uint32, index of each fluid cell; obstacle
// entries are set to 0xffffffff here), adj_out (nFluid*18 uint32, the padded
// SoA PDF index of each link), counts_out[0..1] = nFluid, nCells.
int refh_list_layout(const char *name, const int dims[3], const int periodic[3], int *lattice,
                     int n_kargs, char **kargs, uint32_t *grid_out, uint32_t *adj_out, int *counts_out)
{
	KernelFunctions *kf = refh_find(name);
	if (kf == NULL) return -1;

	LatticeDesc ld;
	refh_fill_ld(&ld, dims, periodic, lattice);

	Parameters p;
	p.nArgs = 0; p.Args = NULL;
	p.nKernelArgs = n_kargs; p.KernelArgs = kargs;

	KernelData *kd = NULL;
	kf->Init(&ld, &kd, &p);
	KernelDataList *kdl = (KernelDataList *)kd;

	size_t n = (size_t)dims[0] * dims[1] * dims[2];
	if (grid_out) {
		for (size_t i = 0; i < n; ++i)
			grid_out[i] = (lattice[i] == LAT_CELL_OBSTACLE) ? 0xffffffffu : kdl->Grid[i];
	}
	if (adj_out) memcpy(adj_out, kdl->AdjList, (size_t)kdl->nFluid * N_D3Q19_IDX * sizeof(uint32_t));
	counts_out[0] = kdl->nFluid;
	counts_out[1] = kdl->nCells;

	kf->Deinit(&ld, &kd);
	return 0;
}
