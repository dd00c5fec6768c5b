/* lbm_main.c -- command-line driver of the B200 kernels (bin/lbmbenchk-b200).
 *
 * Accepts the reference driver's flags (src/Main.c:184-390) and follows its
 * sequence: geometry -> kernel lookup by name (case-insensitive) -> Init ->
 * [-verify initialisation] -> Kernel -> statistics -> [verification] ->
 * metrics -> Deinit, printing the same "P:" result line (src/Main.c:612-627)
 * and the same exit code rule (1 when the -verify error exceeds 0.1,
 * src/Main.c:631-643). Kernels come from liblbmb200.so's table; the CPU
 * kernels of the reference are not part of this build.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "../../include/lbm_b200.h"

static int parse_dims(const char *s, int *d)
{
	const char *p = s;
	for (int i = 0; i < 3; ++i) {
		d[i] = atoi(p);
		if (d[i] <= 0) { printf("ERROR: parameter for %c dimension must be > 0.\n", "XYZ"[i]); return 0; }
		if (i < 2) {
			p = strchr(p, 'x');
			if (!p) { printf("ERROR: parameter for %c dimension is missing.\n", "YZ"[i]); return 0; }
			++p;
		}
	}
	return 1;
}

static void usage(void)
{
	printf("Usage:\n");
	printf("./lbmbenchk-b200 -list\n");
	printf("./lbmbenchk-b200\n");
	printf("      [-dims XxYxZ] [-geometry box|channel|pipe|blocks[-value]|fluid|spheres[:seed:porosity:rmin:rmax]]\n");
	printf("      [-iterations <iterations>] [-rho-in <density>] [-rho-out <density>] [-omega <omega>]\n");
	printf("      [-x-force <force>] [-kernel <kernel>] [-periodic-x] [-periodic-y] [-periodic-z]\n");
	printf("      [-verify] [-vtk [<every-n-iteration>]] [-device <n>] [-t <threads>] [-pin <cores>]\n");
	printf("      -- <kernel specific parameters>\n");
}

int main(int argc, char *argv[])
{
	int dims[3] = { 20, 20, 20 };
	int periodic[3] = { 0, 0, 0 };
	const char *geometry = "channel";
	const char *kernelName = "cuda-list-aa-pv-soa";
	int verify = 0, device = 0;
	CaseData cd;
	memset(&cd, 0, sizeof(cd));
	cd.MaxIterations = 10;
	cd.RhoIn = 1.0; cd.RhoOut = 1.0; cd.Omega = 1.0;
	cd.VtkModulus = 100; cd.StatisticsModulus = 100;
	cd.XForce = 0.00001;
	Parameters p = { argc, argv, 0, NULL };

	printf("# LBM Benchmark Kernels, B200 (sm_100a) build\n");

#define ARG_IS(s) (!strcmp(argv[i], s) || (argv[i][0] == '-' && argv[i][1] == '-' && !strcmp(argv[i] + 1, s)))
#define NEED() do { if (i + 1 >= argc) { printf("ERROR: argument %s requires a parameter.\n", argv[i]); return 1; } } while (0)
	for (int i = 1; i < argc; ++i) {
		if (ARG_IS("-dims")) { NEED(); if (!parse_dims(argv[++i], dims)) return 1; }
		else if (ARG_IS("-geometry")) { NEED(); geometry = argv[++i]; }
		else if (ARG_IS("-iterations")) {
			NEED(); cd.MaxIterations = (int)strtol(argv[++i], NULL, 0);
			if (cd.MaxIterations <= 0) { printf("ERROR: number of iterations must be > 0.\n"); return 1; }
		}
		else if (ARG_IS("-rho-in")) { NEED(); cd.RhoIn = strtod(argv[++i], NULL); }
		else if (ARG_IS("-rho-out")) { NEED(); cd.RhoOut = strtod(argv[++i], NULL); }
		else if (ARG_IS("-omega")) { NEED(); cd.Omega = strtod(argv[++i], NULL); }
		else if (ARG_IS("-x-force")) { NEED(); cd.XForce = strtod(argv[++i], NULL); }
		else if (ARG_IS("-verify")) {
			/* the reference's -verify preset (src/Main.c:232-265) */
			verify = 1;
			cd.Omega = 1.0; cd.RhoIn = 1.0; cd.RhoOut = 1.0;
			geometry = "box";
			dims[0] = dims[1] = dims[2] = 16;
			cd.XForce = 0.00001;
			cd.MaxIterations = 1000;
			periodic[0] = 1; periodic[1] = 1; periodic[2] = 0;
			printf("#\n# VERIFICATION: verifying flow profile of channel flow.\n#\n");
		}
		else if (ARG_IS("-kernel")) { NEED(); kernelName = argv[++i]; }
		else if (ARG_IS("-list")) {
			int n = 0;
			const LbmB200KernelFunctions *t = lbm_b200_kernels(&n);
			printf("Available kernels to benchmark:\n");
			for (int j = 0; j < n; ++j) printf("   %s\n", t[j].Name);
			return 0;
		}
		else if (ARG_IS("-pin") || ARG_IS("-t") || ARG_IS("-threads")) { NEED(); ++i; /* host threads are not used by the GPU kernels */ }
		else if (ARG_IS("-device")) { NEED(); device = atoi(argv[++i]); }
		else if (ARG_IS("-periodic-x")) periodic[0] = 1;
		else if (ARG_IS("-periodic-y")) periodic[1] = 1;
		else if (ARG_IS("-periodic-z")) periodic[2] = 1;
		else if (ARG_IS("-vtk")) {
			/* src/Main.c:266-285: an optional positive number after the flag is the modulus */
			cd.VtkOutput = 1;
			if (i + 1 < argc && atoi(argv[i + 1]) > 0) cd.VtkModulus = atoi(argv[++i]);
		}
		else if (ARG_IS("-statistics")) {
			printf("ERROR: %s is not available in this build.\n", argv[i]);
			return 1;
		}
		else if (ARG_IS("-h") || ARG_IS("-help")) { usage(); return 1; }
		else if (!strcmp(argv[i], "--")) { p.KernelArgs = &argv[++i]; p.nKernelArgs = argc - i; break; }
		else { printf("ERROR: unknown parameter: %s.\n", argv[i]); exit(1); }
	}
#undef ARG_IS
#undef NEED

	if ((uint64_t)19 * dims[0] * dims[1] * dims[2] > ((2LU << 31) - 1)) {
		printf("ERROR: number of PDFs exceed 2^31.\n");
		exit(1);
	}
	if (lbm_b200_set_device(device) != 0) {
		printf("ERROR: cannot use CUDA device %d: %s\n", device, lbm_b200_last_error());
		return 1;
	}

	LatticeDesc ld;
	if (lbm_geo_create(geometry, dims, periodic, &ld) != 0) exit(1);

	printf("# - iterations:        %d\n", cd.MaxIterations);
	printf("# - geometry:\n");
	printf("#   type:              %s\n", ld.Name);
	printf("#   dimensions:        %d x %d x %d (x, y, z)\n", ld.Dims[0], ld.Dims[1], ld.Dims[2]);
	printf("#   nodes total:       % 10d\n", ld.nObst + ld.nFluid);
	printf("#   nodes fluid:       % 10d (including inlet & outlet)\n", ld.nFluid);
	printf("#   nodes obstacles:   % 10d\n", ld.nObst);
	printf("#   periodicity:       x: %d y: %d z: %d\n", ld.PeriodicX, ld.PeriodicY, ld.PeriodicZ);
	printf("# - flow:\n");
	printf("#   omega:             %f\n", cd.Omega);

	int nk = 0;
	const LbmB200KernelFunctions *table = lbm_b200_kernels(&nk);
	const LbmB200KernelFunctions *kf = NULL;
	for (int j = 0; j < nk; ++j)
		if (!strcasecmp(kernelName, table[j].Name)) { kf = &table[j]; break; }
	if (kf == NULL) {
		printf("ERROR: requested kernel \"%s\" not found.\n", kernelName);
		exit(1);
	}
	printf("#\n# - kernel:            %s\n#\n", kf->Name);

	KernelData *kd = NULL;
	kf->Init(&ld, &kd, &p);
	if (verify) {
		lbm_set_initial_density(&ld, kd, &cd);
		lbm_set_initial_velocity(&ld, kd, &cd);
	}
	printf("# starting kernel...\n");
	kd->Kernel(&ld, kd, &cd);

	printf("# iter: %4d   avg density: %e\n", cd.MaxIterations, lbm_density(kd, &ld));
	double errorNorm = -1.0;
	if (verify) {
		errorNorm = lbm_verify(&ld, kd, &cd, 1);
		printf("# Kernel validation: L2 error norm of relative error: %e\n", errorNorm);
	}

	/* the AA kernels run whole even/odd pairs */
	int itersRun = cd.MaxIterations;
	if (strstr(kf->Name, "aa")) itersRun += itersRun % 2;
	const double duration = kd->Duration;
	const double deviceMs = lbm_b200_last_device_ms(kd);
	const double dataVolGByte = kd->LoopBalance * ld.nFluid * (double)itersRun / 1024. / 1024. / 1024.;
	kf->Deinit(&ld, &kd);

	const double perf = (double)ld.nFluid * (double)itersRun / duration / 1.e6;
	printf("#\n# Evaluation Stats\n");
	printf("#   runtype:     \t%s  \n", verify ? "verification" : "benchmark");
	printf("#   runtime:           \t%.3f s\n", duration);
	printf("#   device time:       \t%.3f s\n", deviceMs / 1e3);
	printf("#   iterations:        \t%d  \n", itersRun);
	printf("#   fluid cells:       \t%d \n", ld.nFluid);
	printf("# Derived metrics\n");
	printf("#   MEM data vol.:     \t%.2f GByte\n", dataVolGByte);
	printf("#   MEM bandwidth:     \t%.2f GByte/s\n", dataVolGByte / duration);
	printf("#   performance:       \t%.3f MFLUP/s\n", perf);
	printf("P:   %f MFLUP/s  t: %d  d: %f s  iter: %d  fnodes: %f x1e6  geo: %s  kernel: %s  %s  %s\n",
	       perf, 1, duration, itersRun, ld.nFluid / 1e6, geometry, kernelName, verify ? "VERIFICATION" : "B", "dp");

	int exitCode = 0;
	if (verify) {
		printf("# VERIFICATION: deviation from analytical solution: %e\n", errorNorm);
		if (errorNorm > 0.1) { printf("# VERIFICATION FAILED.\n"); exitCode = 1; }
		else printf("# VERIFICATION SUCCEEDED.\n");
	}
	free(ld.Lattice);
	return exitCode;
}
