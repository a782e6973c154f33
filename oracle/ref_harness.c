/*
 * Reference harness — TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * Compiles the reference's own host and kernel sources unmodified (the Makefile in this
 * directory includes fun_save_to_file.c, fun_DG.c and OpenMP_Function.c from the reference
 * tree at build time; nothing of them is copied here) and replays the set-up and time-loop
 * sequence of DG_leap_Frog_OpenMP.c:main (lines 45-466) with the minimal fixes that make it
 * run on fresh meshes:
 *   A1  the first NeighborNodes call on uninitialised Edge/Neighbor/ibe (:206) is skipped;
 *       it is recomputed after Neighbor_Edge/IBE at :337 exactly as the driver does.
 *   A2  Get_absorb_square fills fewer entries than Get_Absorb_Square_Num counts
 *       (fun_DG.c:260-279 vs 209-220); the filled count is passed to Absorbing_Fun.
 *   A3  Record reads receiver[] with stride 3 (OpenMP_Function.c:67-68) while Get_Receiver
 *       writes stride 2 (fun_DG.c:397-411); this harness records with stride 2.
 *   A5  Edge is zero-initialised (Neighbor_Edge leaves boundary entries unset, fun_DG.c:584).
 *   A11 materials come per element from a file instead of the attribute table (:249-278).
 * Every shot m uses its own Get_Source result (Source_tri = 1 per call, fun_DG.c:284-353)
 * and the source vector of :233-246.  The time loop per shot is :410-459 with snapshot text
 * I/O replaced by binary float64 dumps.
 *
 * Usage: dgref <mesh_prefix> <matrix_dir> <config_file> <out_dir>
 * config_file: "key value" lines — steps, snap_every, n_src, src x z (n_src lines),
 *              n_rec, rec_file (n_rec x 2 float64), mat_file (K x 3 float64: vp vs rho),
 *              dump_setup 0/1, threads, shots_to_run (default n_src), quiet 0/1.
 */
#ifndef N
#define N 2
#endif
#ifndef Np
#define Np 6
#endif
#ifndef TIME
#define TIME 2500
#endif
#ifndef Fp
#define Fp 15
#endif
#ifndef Pi
#define Pi 3.1415
#endif
#ifndef Channel
#define Channel 1
#endif
#ifndef bound_x
#define bound_x 100
#endif
#ifndef bound_z
#define bound_z 100
#endif
#ifndef Source_tri
#define Source_tri 1
#endif
#ifndef model_w
#define model_w 1800
#endif
#ifndef model_h
#define model_h 1800
#endif
#ifndef Process_Num
#define Process_Num 2
#endif

#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include <unistd.h>
#include <sys/types.h>
#include <sys/stat.h>
#include <fcntl.h>
#include <errno.h>
#include <string.h>
#include <sys/time.h>
#include <omp.h>

#include "fun_save_to_file.c"
#include "fun_DG.c"
#include "OpenMP_Function.c"

static double wall(void)
{
	struct timeval tv;
	gettimeofday(&tv, NULL);
	return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

static void dump(const char *dir, const char *name, const void *p, size_t bytes)
{
	char path[4096];
	snprintf(path, sizeof path, "%s/%s.bin", dir, name);
	FILE *f = fopen(path, "wb");
	if (!f) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
	if (bytes && fwrite(p, 1, bytes, f) != bytes) { fprintf(stderr, "short write %s\n", path); exit(2); }
	fclose(f);
}

static void *xcalloc(size_t n, size_t sz)
{
	void *p = calloc(n ? n : 1, sz);
	if (!p) { fprintf(stderr, "out of memory\n"); exit(2); }
	return p;
}

static double *read_f64(const char *path, size_t n)
{
	double *p = xcalloc(n, sizeof(double));
	FILE *f = fopen(path, "rb");
	if (!f || fread(p, sizeof(double), n, f) != n) { fprintf(stderr, "cannot read %s\n", path); exit(2); }
	fclose(f);
	return p;
}

int main(int argc, char **argv)
{
	if (argc != 5) { fprintf(stderr, "usage: %s mesh_prefix matrix_dir config out_dir\n", argv[0]); return 2; }
	const char *prefix = argv[1], *mdir = argv[2], *cfgp = argv[3], *out = argv[4];
	long steps = 100, snap_every = 0, n_src = 0, n_rec = 0, dump_setup = 1, threads = 0, shots_to_run = -1, quiet = 1;
	double src[64][2];
	char rec_file[4096] = "", mat_file[4096] = "";
	{
		FILE *f = fopen(cfgp, "r");
		if (!f) { fprintf(stderr, "cannot open config %s\n", cfgp); return 2; }
		char key[64];
		long si = 0;
		while (fscanf(f, "%63s", key) == 1) {
			if (!strcmp(key, "steps")) fscanf(f, "%ld", &steps);
			else if (!strcmp(key, "snap_every")) fscanf(f, "%ld", &snap_every);
			else if (!strcmp(key, "n_src")) fscanf(f, "%ld", &n_src);
			else if (!strcmp(key, "src")) { if (si < 64) { fscanf(f, "%lf %lf", &src[si][0], &src[si][1]); si++; } }
			else if (!strcmp(key, "n_rec")) fscanf(f, "%ld", &n_rec);
			else if (!strcmp(key, "rec_file")) fscanf(f, "%4095s", rec_file);
			else if (!strcmp(key, "mat_file")) fscanf(f, "%4095s", mat_file);
			else if (!strcmp(key, "dump_setup")) fscanf(f, "%ld", &dump_setup);
			else if (!strcmp(key, "threads")) fscanf(f, "%ld", &threads);
			else if (!strcmp(key, "shots_to_run")) fscanf(f, "%ld", &shots_to_run);
			else if (!strcmp(key, "quiet")) fscanf(f, "%ld", &quiet);
			else { fprintf(stderr, "unknown config key %s\n", key); return 2; }
		}
		fclose(f);
		if (si != n_src || n_src < 1 || n_src > 64) { fprintf(stderr, "bad n_src\n"); return 2; }
	}
	if (shots_to_run < 0) shots_to_run = n_src;
	if (threads > 0) omp_set_num_threads((int)threads);
	if (quiet) { if (!freopen("/dev/null", "w", stdout)) return 2; }

	char path_tri[4096], path_pt[4096], path_nb[4096], p[4096];
	snprintf(path_tri, sizeof path_tri, "%s.ele", prefix);
	snprintf(path_pt, sizeof path_pt, "%s.node", prefix);
	snprintf(path_nb, sizeof path_nb, "%s.neigh", prefix);

	/* precomputed matrices, DG_leap_Frog_OpenMP.c:64-94 */
	static double FeketeNew[Np][2], S1[Np][N + 1], S2[Np][N + 1], S3[Np][N + 1], V[Np][Np], Vb[N + 1][N + 1],
		Vr[Np][Np], Vs[Np][Np], inverV[Np][Np], inverVb[N + 1][N + 1];
#define RD(name, arr, r, c) snprintf(p, sizeof p, "%s/" name ".txt", mdir); ReadDouble(p, *arr, r, c)
	RD("FeketeNew", FeketeNew, Np, 2);
	RD("S1", S1, Np, N + 1);
	RD("S2", S2, Np, N + 1);
	RD("S3", S3, Np, N + 1);
	RD("V", V, Np, Np);
	RD("Vb", Vb, N + 1, N + 1);
	RD("Vr", Vr, Np, Np);
	RD("Vs", Vs, Np, Np);
	RD("inverV", inverV, Np, Np);
	RD("inverVb", inverVb, N + 1, N + 1);
#undef RD

	long Tri = Calculate_Tri(path_tri);
	long Point_Num = Calculate_Point_Num(path_pt);
	long i, j, k, n, num;
	double sum;

	double *Vp = xcalloc(Tri, 8), *Den = xcalloc(Tri, 8), *Miu = xcalloc(Tri, 8), *Lambda = xcalloc(Tri, 8);
	long *Node_Neighbor = xcalloc(Tri * 3 * (N + 1), 8), *Neighbor = xcalloc(Tri * 3, 8), *Edge = xcalloc(Tri * 3, 8);
	long *Edge_flag = xcalloc(Tri * 3, 8);
	double *absorb_fun = xcalloc(Tri * Np, 8);
	long *Neighbor_Mark = xcalloc(Tri * 3, 8);
	long *Series = xcalloc(Process_Num, 8), *Series_order = xcalloc(Process_Num, 8), *Bound_Series = xcalloc(Process_Num, 8);
	long *Triangle_part = xcalloc(Tri, 8);
	double *Jacobi = xcalloc(Tri, 8), *Jacobi_Edge = xcalloc(Tri * 3, 8);
	double *Q = xcalloc(Tri * 30, 8), *A = xcalloc(Tri * 5, 8), *B = xcalloc(Tri * 5, 8);
	double *Dx = xcalloc(Tri * Np * Np, 8), *Dz = xcalloc(Tri * Np * Np, 8);
	double *S = xcalloc(3 * Np * (N + 1), 8);
	long *ibe = xcalloc(3 * (N + 1), 8);
	double *normal1 = xcalloc(Tri * 2, 8), *normal2 = xcalloc(Tri * 2, 8), *normal3 = xcalloc(Tri * 2, 8);
	double *fun = xcalloc(n_src * Np, 8);
	double *Point = xcalloc(Point_Num * 2, 8);
	long *Triangle = xcalloc(Tri * 3, 8), *neighbor = xcalloc(Tri * 3, 8), *attribute = xcalloc(Tri, 8);

	Mesh_Input(Tri, Point_Num, path_tri, path_nb, path_pt, Point, Triangle, neighbor, attribute);
	/* A1: the uninitialised NeighborNodes call of :206 is skipped */
	long *epart = xcalloc(Tri, 8); /* single partition: element order does not affect results */

	Normals(Tri, Point, Triangle, normal1, normal2, normal3);
	Jacobian(Tri, Jacobi_Edge, Jacobi, Point, Triangle);

	long *source = xcalloc(n_src * 2, 8);
	for (long m = 0; m < n_src; m++) {
		long s1[2] = {0, 0};
		Get_Source(Tri, Point_Num, Point, Triangle, s1, src[m]);
		source[m * 2 + 0] = s1[0];
		source[m * 2 + 1] = s1[1];
	}
	long *receiver = xcalloc(n_rec * 2 + 2, 8);
	double *rec_pos = n_rec ? read_f64(rec_file, n_rec * 2) : NULL;
	for (long r = 0; r < n_rec; r++) {
		long r1[2] = {0, 0};
		Get_Receiver(Tri, Point_Num, Point, Triangle, r1, &rec_pos[r * 2]);
		receiver[r * 2 + 0] = r1[0];
		receiver[r * 2 + 1] = r1[1];
	}

	/* source vector of :233-246 per shot */
	for (long m = 0; m < n_src; m++) {
		for (i = 0; i < Np; i++) {
			n = source[m * 2 + 0] - 1;
			k = source[m * 2 + 1] - 1;
			sum = 0;
			for (j = 0; j < Np; j++)
				sum = sum + V[i][j] * V[k][j];
			fun[m * Np + i] = sum / Jacobi[n];
		}
	}

	/* materials per element (A11), formulas of :252-253 */
	{
		double *mat = read_f64(mat_file, Tri * 3);
		for (i = 0; i < Tri; i++) {
			double Cp = mat[i * 3 + 0], Cs = mat[i * 3 + 1], den = mat[i * 3 + 2];
			double miu = den * Cs * Cs;
			double lambda = den * Cp * Cp - 2 * miu;
			Vp[i] = Cp;
			Lambda[i] = lambda;
			Miu[i] = miu;
			Den[i] = den;
		}
		free(mat);
	}

	double dt = Calculate_Time_Step(Tri, Point, Triangle, Vp);
	double t0 = Ricker_Delay_Time(dt);

	long Absorb_Num = Get_Absorb_Square_Num(Tri, Point, Triangle);
	long Inside_Num = Get_Inside_Square_Num(Tri, Point, Triangle);
	long *absorbing_triangle = xcalloc(Absorb_Num, 8);
	long *inside_triangle = xcalloc(Inside_Num, 8);
	Get_absorb_square(Tri, Point, Triangle, absorbing_triangle, inside_triangle);
	long filled = 0; /* A2 */
	while (filled < Absorb_Num && absorbing_triangle[filled] != 0)
		filled++;
	Absorbing_Fun(Tri, filled, 0.1, absorb_fun, absorbing_triangle, Point, Triangle, FeketeNew);

	Elastic_A_B(Tri, A, B, Lambda, Miu, Den);
	for (j = 0; j < Np; j++)
		for (n = 0; n < N + 1; n++) {
			S[0 * Np * (N + 1) + j * (N + 1) + n] = S1[j][n];
			S[1 * Np * (N + 1) + j * (N + 1) + n] = S2[j][n];
			S[2 * Np * (N + 1) + j * (N + 1) + n] = S3[j][n];
		}
	long *neighbor_in = xcalloc(Tri * 3, 8);
	memcpy(neighbor_in, neighbor, Tri * 3 * 8);
	Neighbor_Edge(Tri, Neighbor, neighbor, Edge, Triangle, Edge_flag);
	IBE(ibe);
	NeighborNodes(Tri, Node_Neighbor, Triangle, Edge, Neighbor, ibe);
	Dx_Dz(Tri, Dx, Dz, Vr, Vs, inverV, Triangle, Point);
	Neighbor_Partition_Mark(Tri, Neighbor, epart, Neighbor_Mark);
	long Boundary_Num = Calculate_Boundary_Num(Tri, Neighbor_Mark);
	long *Boundary_Triangle = xcalloc(Boundary_Num + 1, 8);
	Partition_Boundary_Neighbor(Tri, Neighbor, epart, Neighbor_Mark, Series, Series_order, Bound_Series, Triangle_part, Boundary_Triangle);
	Central_flux(Tri, Jacobi, Jacobi_Edge, Q, A, B, normal1, normal2, normal3);

	if (dump_setup) {
		long sizes[4] = {Tri, Point_Num, Absorb_Num, filled};
		dump(out, "sizes", sizes, sizeof sizes);
		double scal[2] = {dt, t0};
		dump(out, "dt_t0", scal, sizeof scal);
		dump(out, "Point", Point, Point_Num * 2 * 8);
		dump(out, "Triangle", Triangle, Tri * 3 * 8);
		dump(out, "neighbor_in", neighbor_in, Tri * 3 * 8);
		dump(out, "attribute", attribute, Tri * 8);
		dump(out, "Neighbor", Neighbor, Tri * 3 * 8);
		dump(out, "Edge", Edge, Tri * 3 * 8);
		dump(out, "Edge_flag", Edge_flag, Tri * 3 * 8);
		dump(out, "Node_Neighbor", Node_Neighbor, Tri * 9 * 8);
		dump(out, "ibe", ibe, 9 * 8);
		dump(out, "Jacobi", Jacobi, Tri * 8);
		dump(out, "Jacobi_Edge", Jacobi_Edge, Tri * 3 * 8);
		dump(out, "normal1", normal1, Tri * 2 * 8);
		dump(out, "normal2", normal2, Tri * 2 * 8);
		dump(out, "normal3", normal3, Tri * 2 * 8);
		dump(out, "A", A, Tri * 5 * 8);
		dump(out, "B", B, Tri * 5 * 8);
		dump(out, "Q", Q, Tri * 30 * 8);
		dump(out, "Dx", Dx, Tri * 36 * 8);
		dump(out, "Dz", Dz, Tri * 36 * 8);
		dump(out, "S", S, 54 * 8);
		dump(out, "absorb_fun", absorb_fun, Tri * Np * 8);
		dump(out, "absorbing_triangle", absorbing_triangle, Absorb_Num * 8);
		dump(out, "source", source, n_src * 2 * 8);
		dump(out, "fun", fun, n_src * Np * 8);
		dump(out, "receiver", receiver, n_rec * 2 * 8);
		dump(out, "Vp", Vp, Tri * 8);
		double mats[4][1];
		(void)mats;
		double ops[6 * 6 * 4 + 6 * 2];
		memcpy(ops, Vr, 288); memcpy(ops + 36, Vs, 288); memcpy(ops + 72, inverV, 288); memcpy(ops + 108, V, 288);
		memcpy(ops + 144, FeketeNew, 96);
		dump(out, "ops_Vr_Vs_inverV_V_Fekete", ops, sizeof ops);
	}

	/* time loop, :395-459 */
	double *Vx1 = xcalloc(Tri * Np, 8), *Vz1 = xcalloc(Tri * Np, 8), *Txx1 = xcalloc(Tri * Np, 8),
		*Tzz1 = xcalloc(Tri * Np, 8), *Txz1 = xcalloc(Tri * Np, 8);
	double *rec_x = xcalloc(steps * (n_rec ? n_rec : 1), 8), *rec_z = xcalloc(steps * (n_rec ? n_rec : 1), 8);
	double loop_seconds = 0.0;
	for (long m = 0; m < shots_to_run; m++) {
		memset(Vx1, 0, sizeof(double) * Np * Tri);
		memset(Vz1, 0, sizeof(double) * Np * Tri);
		memset(Txx1, 0, sizeof(double) * Np * Tri);
		memset(Tzz1, 0, sizeof(double) * Np * Tri);
		memset(Txz1, 0, sizeof(double) * Np * Tri);
		double start = wall();
		for (long time = 0; time < steps; time++) {
			double w = Ricker_Source(time, dt, t0);
			Absorb_Boundary(Tri, Vx1, Vz1, Txx1, Tzz1, Txz1, absorb_fun, Triangle_part, Series, Series_order);
			source_kernel(Vz1, source, fun, w, m);
			LU_Velocity(Tri, dt, Vx1, Vz1, Txx1, Tzz1, Txz1, Triangle_part, Neighbor_Mark, Series, Series_order, A, B, Dx, Dz, Q, S, ibe, Node_Neighbor, Neighbor, Edge_flag);
			LU_Stress_Elastic(Tri, dt, Txx1, Tzz1, Txz1, Vx1, Vz1, Triangle_part, Neighbor_Mark, Series, Series_order, A, B, Dx, Dz, Q, S, ibe, Node_Neighbor, Neighbor, Edge_flag);
			for (long r = 0; r < n_rec; r++) { /* A3: stride 2 */
				long rt = receiver[r * 2 + 0], rn = receiver[r * 2 + 1];
				rec_x[time * n_rec + r] = Vx1[Np * (rt - 1) + rn - 1];
				rec_z[time * n_rec + r] = Vz1[Np * (rt - 1) + rn - 1];
			}
			if (snap_every > 0 && (time + 1) % snap_every == 0) {
				double t_io = wall();
				char name[128];
				snprintf(name, sizeof name, "shot%ld_Vx%ld", m, time + 1);
				dump(out, name, Vx1, Tri * Np * 8);
				snprintf(name, sizeof name, "shot%ld_Vz%ld", m, time + 1);
				dump(out, name, Vz1, Tri * Np * 8);
				start += wall() - t_io; /* snapshot I/O is not loop time */
			}
		}
		loop_seconds += wall() - start;
		char name[128];
		snprintf(name, sizeof name, "shot%ld_rec_x", m);
		dump(out, name, rec_x, steps * n_rec * 8);
		snprintf(name, sizeof name, "shot%ld_rec_z", m);
		dump(out, name, rec_z, steps * n_rec * 8);
		const char *fn[5] = {"Vx", "Vz", "Txx", "Tzz", "Txz"};
		double *fp[5] = {Vx1, Vz1, Txx1, Tzz1, Txz1};
		for (int q = 0; q < 5; q++) {
			snprintf(name, sizeof name, "shot%ld_final_%s", m, fn[q]);
			dump(out, name, fp[q], Tri * Np * 8);
		}
	}
	{
		FILE *f;
		char tp[4096];
		snprintf(tp, sizeof tp, "%s/timing.txt", out);
		f = fopen(tp, "w");
		if (f) {
			fprintf(f, "loop_seconds %.9f\nthreads %d\nK %ld\nsteps %ld\nshots %ld\n", loop_seconds,
					omp_get_max_threads(), Tri, steps, shots_to_run);
			fclose(f);
		}
	}
	return 0;
}
