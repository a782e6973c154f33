/*
 * dg_oracle.c — CPU ORACLE, TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's per-step time loop, used by the tests (and the
 * benchmark's CPU-baseline leg) as the checker for the GPU engine.  It is never linked into
 * the product.  Parity is pinned: its traces and fields equal, bit for bit, those of the
 * reference's own OpenMP code compiled from the reference sources (oracle/_ref) on the golden
 * fixtures under tests/golden.
 *
 * One step, in the reference order (DG_leap_Frog_OpenMP.c:418-437):
 *   sponge      every field *= absorb_fun                 OpenMP_Function.c:25-46
 *   source      Vz[src] += fun * w(t)                     OpenMP_Function.c:49-58
 *   velocity    V += dt * L_V(T)                          OpenMP_Function.c:75-185
 *   stress      T += dt * L_T(V)                          OpenMP_Function.c:188-306
 *   record      rec[t][r] = V at (triangle, node)         OpenMP_Function.c:61-72 (stride 2)
 * Arithmetic keeps the reference's operation order; build with -ffp-contract=off.
 * Arrays are the reference's: element-major fields (value i of element e at [e*6+i]),
 * 1-based int64 maps.
 */
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
#define DGO_HAVE_MXCSR 1
#endif

/*
 * Subnormal mode of dgo_run (dgo_set_flush_subnormals): off by default, the arithmetic of the
 * reference.  On, the threads of each loop flush subnormal results and operands to zero
 * (x86 MXCSR FTZ and DAZ) for the loop's duration, then restore their mode.  Values below 2^-1022
 * ahead of the wave front then become 0 and the host no longer slows down several times as they
 * spread; every other value changes by less than 2^-1022 in absolute terms.  Only for long runs
 * compared against the GPU at a relative tolerance; never for a bit-exact comparison.
 */
static int g_flush = 0;
#ifdef DGO_HAVE_MXCSR
#define DGO_MODE_ENTER unsigned dgo_csr_ = _mm_getcsr(); if (g_flush) _mm_setcsr(dgo_csr_ | 0x8040u);
#define DGO_MODE_LEAVE _mm_setcsr(dgo_csr_);
#else
#define DGO_MODE_ENTER
#define DGO_MODE_LEAVE
#endif

void dgo_set_flush_subnormals(int on) { g_flush = on != 0; }

#define NP 6
#define NF 3

typedef struct {
	long K;
	const double *A, *B;         /* [K][5] */
	const double *Dx, *Dz;       /* [K][6][6] */
	const double *Q;             /* [K][3][5][2] */
	const double *S;             /* [3][6][3] */
	const long *ibe;             /* [3][3] 1-based */
	const long *Node_Neighbor;   /* [K][3][3] 1-based */
	const long *Neighbor;        /* [K][3] 1-based */
	const long *Edge_flag;       /* [K][3] */
	const double *absorb_fun;    /* [K][6] */
	const long *source;          /* [shots][2] */
	const double *fun;           /* [shots][6] */
	long n_rec;
	const long *receiver;        /* [n_rec][2] stride 2 */
	double dt;
	const double *wavelet;       /* [n_steps] */
	long n_steps;
} dgo_problem;

/* one element of the velocity half-step (OpenMP_Function.c:106-182) */
static void velocity_element(const dgo_problem *p, long e, double *Vx, double *Vz, const double *Txx,
							 const double *Tzz, const double *Txz)
{
	const double *dx = p->Dx + e * 36, *dz = p->Dz + e * 36;
	const double *own_xx = Txx + e * NP, *own_zz = Tzz + e * NP, *own_xz = Txz + e * NP;
	double vol_x[NP], vol_z[NP], fx[NF][NP], fz[NF][NP];
	for (int i = 0; i < NP; i++) {
		double a = 0, b = 0, c = 0, d = 0;
		for (int n = 0; n < NP; n++) {
			a += dx[i * NP + n] * own_xx[n];
			b += dx[i * NP + n] * own_xz[n];
			c += dz[i * NP + n] * own_zz[n];
			d += dz[i * NP + n] * own_xz[n];
		}
		vol_x[i] = p->A[e * 5 + 0] * a + p->B[e * 5 + 0] * d;
		vol_z[i] = p->A[e * 5 + 1] * b + p->B[e * 5 + 1] * c;
	}
	for (int f = 0; f < 3; f++) {
		const long nb = p->Neighbor[e * 3 + f] - 1;
		const double flag = (double)p->Edge_flag[e * 3 + f];
		double jxx[NF], jzz[NF], jxz[NF];
		for (int k = 0; k < NF; k++) {
			const long there = NP * nb + p->Node_Neighbor[e * 9 + f * 3 + k] - 1;
			const long here = NP * e + p->ibe[f * 3 + k] - 1;
			jxx[k] = Txx[there] * flag - Txx[here];
			jzz[k] = Tzz[there] * flag - Tzz[here];
			jxz[k] = Txz[there] * flag - Txz[here];
		}
		const double *S = p->S + f * NP * NF;
		const double *q = p->Q + e * 30 + f * 10;
		for (int i = 0; i < NP; i++) {
			double lxx = 0, lzz = 0, lxz = 0;
			for (int k = 0; k < NF; k++) {
				lxx += S[i * NF + k] * jxx[k];
				lzz += S[i * NF + k] * jzz[k];
				lxz += S[i * NF + k] * jxz[k];
			}
			fx[f][i] = q[0] * lxx + q[1] * lxz;
			fz[f][i] = q[2] * lzz + q[3] * lxz;
		}
	}
	for (int i = 0; i < NP; i++) {
		Vx[e * NP + i] = (vol_x[i] + fx[0][i] + fx[1][i] + fx[2][i]) * p->dt + Vx[e * NP + i];
		Vz[e * NP + i] = (vol_z[i] + fz[0][i] + fz[1][i] + fz[2][i]) * p->dt + Vz[e * NP + i];
	}
}

/* one element of the stress half-step (OpenMP_Function.c:227-303) */
static void stress_element(const dgo_problem *p, long e, double *Txx, double *Tzz, double *Txz, const double *Vx,
						   const double *Vz)
{
	const double *dx = p->Dx + e * 36, *dz = p->Dz + e * 36;
	const double *own_x = Vx + e * NP, *own_z = Vz + e * NP;
	double vxx[NP], vzz[NP], vxz[NP], f_xx[NF][NP], f_zz[NF][NP], f_xz[NF][NP];
	const double *A = p->A + e * 5, *B = p->B + e * 5;
	for (int i = 0; i < NP; i++) {
		double dxvx = 0, dxvz = 0, dzvx = 0, dzvz = 0;
		for (int n = 0; n < NP; n++) {
			dxvx += dx[i * NP + n] * own_x[n];
			dxvz += dx[i * NP + n] * own_z[n];
			dzvx += dz[i * NP + n] * own_x[n];
			dzvz += dz[i * NP + n] * own_z[n];
		}
		vxx[i] = A[2] * dxvx + B[2] * dzvz;
		vzz[i] = A[3] * dxvx + B[3] * dzvz;
		vxz[i] = A[4] * dxvz + B[4] * dzvx;
	}
	for (int f = 0; f < 3; f++) {
		const long nb = p->Neighbor[e * 3 + f] - 1;
		const double flag = (double)p->Edge_flag[e * 3 + f];
		double jx[NF], jz[NF];
		for (int k = 0; k < NF; k++) {
			const long there = NP * nb + p->Node_Neighbor[e * 9 + f * 3 + k] - 1;
			const long here = NP * e + p->ibe[f * 3 + k] - 1;
			jx[k] = Vx[there] * flag - Vx[here];
			jz[k] = Vz[there] * flag - Vz[here];
		}
		const double *S = p->S + f * NP * NF;
		const double *q = p->Q + e * 30 + f * 10;
		for (int i = 0; i < NP; i++) {
			double lx = 0, lz = 0;
			for (int k = 0; k < NF; k++) {
				lx += S[i * NF + k] * jx[k];
				lz += S[i * NF + k] * jz[k];
			}
			f_xx[f][i] = q[4] * lx + q[5] * lz;
			f_zz[f][i] = q[6] * lx + q[7] * lz;
			f_xz[f][i] = q[8] * lx + q[9] * lz;
		}
	}
	for (int i = 0; i < NP; i++) {
		const long o = e * NP + i;
		Txx[o] = (vxx[i] + f_xx[0][i] + f_xx[1][i] + f_xx[2][i]) * p->dt + Txx[o];
		Tzz[o] = (vzz[i] + f_zz[0][i] + f_zz[1][i] + f_zz[2][i]) * p->dt + Tzz[o];
		Txz[o] = (vxz[i] + f_xz[0][i] + f_xz[1][i] + f_xz[2][i]) * p->dt + Txz[o];
	}
}

/*
 * Advance the five fields of shot `shot` from step t_begin for `steps` steps.  rec_x/rec_z
 * receive [steps][n_rec] samples (may be NULL).  threads <= 0 keeps the OpenMP default.
 */
int dgo_run(const dgo_problem *p, long shot, long t_begin, long steps, double *Vx, double *Vz, double *Txx,
			double *Tzz, double *Txz, double *rec_x, double *rec_z, int threads)
{
	if (!p || !Vx || !Vz || !Txx || !Tzz || !Txz || steps < 0 || t_begin < 0 || t_begin + steps > p->n_steps)
		return -1;
	const long K = p->K, KN = p->K * NP;
#ifdef _OPENMP
	if (threads > 0) omp_set_num_threads(threads);
#else
	(void)threads;
#endif
	for (long t = t_begin; t < t_begin + steps; t++) {
		const double w = p->wavelet[t];
#pragma omp parallel
		{
			DGO_MODE_ENTER
#pragma omp for schedule(static)
			for (long id = 0; id < KN; id++) {
				const double a = p->absorb_fun[id];
				Vx[id] *= a;
				Vz[id] *= a;
				Txx[id] *= a;
				Tzz[id] *= a;
				Txz[id] *= a;
			}
#pragma omp single
			for (int i = 0; i < NP; i++)
				Vz[NP * (p->source[shot * 2 + 0] - 1) + i] += p->fun[shot * NP + i] * w;
#pragma omp for schedule(static)
			for (long e = 0; e < K; e++)
				velocity_element(p, e, Vx, Vz, Txx, Tzz, Txz);
#pragma omp for schedule(static)
			for (long e = 0; e < K; e++)
				stress_element(p, e, Txx, Tzz, Txz, Vx, Vz);
			DGO_MODE_LEAVE
		}
		if (rec_x && rec_z)
			for (long r = 0; r < p->n_rec; r++) {
				const long at = NP * (p->receiver[r * 2 + 0] - 1) + p->receiver[r * 2 + 1] - 1;
				rec_x[(t - t_begin) * p->n_rec + r] = Vx[at];
				rec_z[(t - t_begin) * p->n_rec + r] = Vz[at];
			}
	}
	return 0;
}

/*
 * One half of step t, for the test of a mesh split into parts (the halves of dgo_run's step with
 * an exchange of ghost values in between): half 0 = sponge on all fields, source, velocity
 * update; half 1 = stress update and the record of step t into rec_x/rec_z[n_rec] (may be NULL).
 */
int dgo_half(const dgo_problem *p, long shot, long t, int half, double *Vx, double *Vz, double *Txx, double *Tzz,
			 double *Txz, double *rec_x, double *rec_z)
{
	if (!p || !Vx || !Vz || !Txx || !Tzz || !Txz || t < 0 || t >= p->n_steps || (half != 0 && half != 1))
		return -1;
	const long K = p->K, KN = p->K * NP;
	if (half == 0) {
		const double w = p->wavelet[t];
		for (long id = 0; id < KN; id++) {
			const double a = p->absorb_fun[id];
			Vx[id] *= a;
			Vz[id] *= a;
			Txx[id] *= a;
			Tzz[id] *= a;
			Txz[id] *= a;
		}
		for (int i = 0; i < NP; i++)
			Vz[NP * (p->source[shot * 2 + 0] - 1) + i] += p->fun[shot * NP + i] * w;
		for (long e = 0; e < K; e++)
			velocity_element(p, e, Vx, Vz, Txx, Tzz, Txz);
		return 0;
	}
	for (long e = 0; e < K; e++)
		stress_element(p, e, Txx, Tzz, Txz, Vx, Vz);
	if (rec_x && rec_z)
		for (long r = 0; r < p->n_rec; r++) {
			const long at = NP * (p->receiver[r * 2 + 0] - 1) + p->receiver[r * 2 + 1] - 1;
			rec_x[r] = Vx[at];
			rec_z[r] = Vz[at];
		}
	return 0;
}

int dgo_max_threads(void)
{
#ifdef _OPENMP
	return omp_get_max_threads();
#else
	return 1;
#endif
}
