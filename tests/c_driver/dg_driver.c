/*
 * A C driver of the engine, written the way the reference's C time loop would call it
 * (test of the C ABI from C: the header is C99, the structs and calls line up, snapshots come
 * back through a C callback).
 *
 *   dg_driver <in_dir> <precision 0..3> <steps> <every> <out_dir>
 *
 * <in_dir> holds the set-up arrays as raw little-endian files (doubles, or int64 for the index
 * maps) and sizes.txt = "K n_points n_shots n_rec n_steps dt".  The driver steps `steps` steps
 * with a Vx/Vz snapshot of shot 0 every `every` steps (dg_gpu_step_snapshots), then writes
 * trace_x.bin / trace_z.bin of shot 0, the final Txz of shot 0 and the snapshots to <out_dir>.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dg_gpu.h"

static void *load(const char *dir, const char *name, size_t bytes)
{
	char path[1024];
	snprintf(path, sizeof path, "%s/%s.bin", dir, name);
	FILE *f = fopen(path, "rb");
	if (!f) return NULL;
	void *p = malloc(bytes ? bytes : 1);
	size_t got = p ? fread(p, 1, bytes, f) : 0;
	fclose(f);
	if (got != bytes) { free(p); return NULL; }
	return p;
}

static int save(const char *dir, const char *name, const double *v, size_t n)
{
	char path[1024];
	snprintf(path, sizeof path, "%s/%s.bin", dir, name);
	FILE *f = fopen(path, "wb");
	if (!f) return 1;
	size_t put = fwrite(v, sizeof(double), n, f);
	fclose(f);
	return put != n;
}

struct snaps { double *all; long K; long count; };

static void on_snapshot(void *user, long step, const double *vx, const double *vz)
{
	struct snaps *s = (struct snaps *)user;
	(void)step;
	memcpy(s->all + s->count * 2 * s->K * 6, vx, sizeof(double) * s->K * 6);
	memcpy(s->all + (s->count * 2 + 1) * s->K * 6, vz, sizeof(double) * s->K * 6);
	s->count++;
}

int main(int argc, char **argv)
{
	if (argc != 6) { fprintf(stderr, "usage: dg_driver in_dir precision steps every out_dir\n"); return 2; }
	const char *in = argv[1], *out = argv[5];
	const int precision = atoi(argv[2]);
	const long steps = atol(argv[3]), every = atol(argv[4]);
	char path[1024];
	snprintf(path, sizeof path, "%s/sizes.txt", in);
	FILE *f = fopen(path, "r");
	long K, P, S, R, T;
	double dt;
	if (!f || fscanf(f, "%ld %ld %ld %ld %ld %lf", &K, &P, &S, &R, &T, &dt) != 6) { fprintf(stderr, "sizes\n"); return 2; }
	fclose(f);

	dg_gpu_mesh m;
	memset(&m, 0, sizeof m);
	m.K = K; m.Np = 6; m.Nfp = 3; m.n_points = P;
	m.Point = load(in, "Point", sizeof(double) * P * 2);
	m.Triangle = load(in, "Triangle", sizeof(long) * K * 3);
	m.Vr = load(in, "Vr", sizeof(double) * 36);
	m.Vs = load(in, "Vs", sizeof(double) * 36);
	m.inverV = load(in, "inverV", sizeof(double) * 36);
	m.V = load(in, "V", sizeof(double) * 36);
	m.S = load(in, "S", sizeof(double) * 54);
	m.ibe = load(in, "ibe", sizeof(long) * 9);
	m.Neighbor = load(in, "Neighbor", sizeof(long) * K * 3);
	m.Node_Neighbor = load(in, "Node_Neighbor", sizeof(long) * K * 9);
	m.Edge_flag = load(in, "Edge_flag", sizeof(long) * K * 3);
	m.A = load(in, "A", sizeof(double) * K * 5);
	m.B = load(in, "B", sizeof(double) * K * 5);
	m.Dx = load(in, "Dx", sizeof(double) * K * 36);
	m.Dz = load(in, "Dz", sizeof(double) * K * 36);
	m.Q = load(in, "Q", sizeof(double) * K * 30);
	m.absorb_fun = load(in, "absorb_fun", sizeof(double) * K * 6);
	m.n_shots = (int)S;
	m.source = load(in, "source", sizeof(long) * S * 2);
	m.fun = load(in, "fun", sizeof(double) * S * 6);
	m.n_rec = (int)R;
	m.receiver = load(in, "receiver", sizeof(long) * R * 2);
	m.dt = dt;
	m.n_steps = T;
	m.wavelet = load(in, "wavelet", sizeof(double) * T);
	if (!m.Point || !m.Triangle || !m.Neighbor || !m.A || !m.wavelet || !m.source || !m.receiver) {
		fprintf(stderr, "missing input arrays\n");
		return 2;
	}

	dg_gpu_opts o;
	dg_gpu_default_opts(&o);
	o.precision = precision;
	dg_gpu_ctx *ctx = NULL;
	int rc = dg_gpu_init(&ctx, &m, 1, &o);
	if (rc) { fprintf(stderr, "dg_gpu_init: %s (%s)\n", dg_gpu_strerror(rc), dg_gpu_last_error()); return 1; }

	struct snaps sn;
	sn.K = K;
	sn.count = 0;
	sn.all = malloc(sizeof(double) * (size_t)(steps / every) * 2 * K * 6 + 1);
	rc = dg_gpu_step_snapshots(ctx, steps, every, 0, 0, on_snapshot, &sn);
	if (rc) { fprintf(stderr, "dg_gpu_step_snapshots: %s (%s)\n", dg_gpu_strerror(rc), dg_gpu_last_error()); return 1; }

	double *tx = malloc(sizeof(double) * steps * R + 1), *tz = malloc(sizeof(double) * steps * R + 1);
	double *txz = malloc(sizeof(double) * K * 6);
	if (dg_gpu_fetch(ctx, DG_TRACE_X, 0, 0, tx) || dg_gpu_fetch(ctx, DG_TRACE_Z, 0, 0, tz) ||
		dg_gpu_fetch(ctx, DG_TXZ, 0, 0, txz)) {
		fprintf(stderr, "dg_gpu_fetch: %s\n", dg_gpu_last_error());
		return 1;
	}
	dg_gpu_stats st;
	dg_gpu_stats_get(ctx, &st);
	rc = save(out, "trace_x", tx, steps * R) | save(out, "trace_z", tz, steps * R) | save(out, "Txz", txz, K * 6) |
		 save(out, "snapshots", sn.all, sn.count * 2 * K * 6);
	printf("steps %ld snapshots %ld family %d\n", st.steps_done, sn.count, st.kernel_family);

	/* the same steps again as half steps in two parts (no ghosts here, so every element is in
	 * the interior part), the parts in both orders, with an enqueue-only pack of the (empty)
	 * send list on the context's stream */
	int rp = dg_gpu_reset(ctx);
	if (!rp && !dg_gpu_context_stream(ctx)) rp = -1;
	if (!rp) rp = dg_gpu_halo_lists(ctx, 0, 0, NULL, 0, NULL);
	for (long t = 0; t < steps && !rp; t++) {
		rp = dg_gpu_half_step_part(ctx, 0, DG_PART_INTERIOR);
		if (!rp) rp = dg_gpu_half_step_part(ctx, 0, DG_PART_BOUNDARY);
		if (!rp) rp = dg_gpu_halo_pack_async(ctx, 0, 0, NULL);
		if (!rp) rp = dg_gpu_half_step_part(ctx, 1, DG_PART_BOUNDARY);
		if (!rp) rp = dg_gpu_half_step_part(ctx, 1, DG_PART_INTERIOR);
	}
	if (!rp) rp = dg_gpu_fetch(ctx, DG_TXZ, 0, 0, txz);
	if (rp) {
		fprintf(stderr, "half steps in parts: %s (%s)\n", dg_gpu_strerror(rp), dg_gpu_last_error());
		return 1;
	}
	rc |= save(out, "Txz_parts", txz, K * 6);
	dg_gpu_free(ctx);
	return rc;
}
