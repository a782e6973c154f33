/*
 * dg_host.c — host set-up of the DG time loop (see include/dg_host.h for the function map).
 *
 * Floating-point expressions keep the reference's evaluation order and its libm calls
 * (pow, sqrt, acos, cos, exp) so that, compiled with -ffp-contract=off, every array equals
 * what fun_DG.c produces.  Comments give the reference lines each block follows.
 *
 * Per-element loops run on OpenMP threads: each element's values depend on that element alone,
 * and the reductions over elements (the smallest inscribed radius, counts) are evaluated in
 * element order after the parallel loop, so the arrays do not depend on the thread count.
 */
#include "dg_host.h"

#include <fcntl.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#define NPN 6 /* nodes per P2 triangle */
#define NFN 3 /* nodes per face */

const char *dgh_strerror(int code)
{
	switch (code) {
	case DGH_OK: return "ok";
	case DGH_ERR_IO: return "cannot open or read file";
	case DGH_ERR_FORMAT: return "file holds fewer values than requested or a malformed number";
	case DGH_ERR_ARG: return "invalid argument";
	case DGH_ERR_NOSOURCE: return "source position does not coincide with a mesh vertex";
	case DGH_ERR_NORECEIVER: return "receiver position does not coincide with a mesh vertex";
	case DGH_ERR_MESH: return "invalid mesh (vertex index out of range or repeated vertex)";
	case DGH_ERR_NOMEM: return "out of memory";
	default: return "unknown error";
	}
}

/* ---------------------------------------------------------------- text numbers ---------- */

/* pow(10, k) for k = -99..99 (the exponents two digits can write), filled by libm's pow itself,
 * so a table lookup returns exactly what the reference's pow calls return. */
typedef struct { double v[199]; } pow10_table;
static void pow10_fill(pow10_table *t)
{
	for (int k = -99; k <= 99; k++) t->v[k + 99] = pow(10, k);
}
static inline double p10(const pow10_table *t, long k) { return (k >= -99 && k <= 99) ? t->v[k + 99] : pow(10, k); }

/* ReadDouble's per-token arithmetic (fun_save_to_file.c:63-93): leading digit, then the seven
 * fraction digits added from the last one upwards with pow(10, k), then the power of ten and
 * the sign applied in that order. */
static double parse_e7(const char *s, long i, const pow10_table *t)
{
	double sign = 1.0, esign = 1.0, v;
	long k, j, p;
	if (s[i - 10] == '-') sign = -1.0;
	if (s[i + 1] == '-') esign = -1.0;
	v = (double)(s[i - 9] - '0');
	for (j = i - 1, k = -7; j >= i - 7; j--, k++)
		v = v + (s[j] - '0') * p10(t, k);
	p = (long)esign * ((s[i + 2] - '0') * 10 + (s[i + 3] - '0'));
	return v * p10(t, p) * sign;
}

double dgh_parse_e7(const char *s, long i)
{
	pow10_table t;
	pow10_fill(&t);
	return parse_e7(s, i, &t);
}

/* ReadInt's per-token arithmetic (fun_save_to_file.c:157-185): the signed leading digit times
 * 10^p, then `p` further digits added as positive integer places.  (A negative number with
 * more than one significant digit therefore comes out wrong in the reference; -1, the only
 * negative value the mesh files hold, is exact.) */
static long parse_int_e7(const char *s, long i, const pow10_table *t)
{
	long sign = 1, esign = 1, p, j, k, v;
	if (s[i - 10] == '-') sign = -1;
	if (s[i + 1] == '-') esign = -1;
	p = esign * ((s[i + 2] - '0') * 10 + (s[i + 3] - '0'));
	v = (long)((s[i - 9] - '0') * p10(t, p) * sign);
	for (j = i - 7, k = p - 1; j <= i - 7 + p - 1; j++, k--)
		v = (long)(v + (s[j] - '0') * p10(t, k));
	return v;
}

void dgh_quantize_e7(double *x, long n)
{
	pow10_table t;
	pow10_fill(&t);
#pragma omp parallel for schedule(static)
	for (long q = 0; q < n; q++) {
		char buf[64];
		int len = snprintf(buf + 8, sizeof buf - 8, "%16.7e", x[q]);
		memset(buf, ' ', 8);
		char *e = strchr(buf + 8, 'e');
		if (len <= 0 || !e || e - buf < 10 || !isfinite(x[q]))
			continue;
		x[q] = parse_e7(buf, (long)(e - buf), &t);
	}
}

/* The file (or its first `limit` bytes, limit > 0), with 16 bytes of padding on each side so
 * s[i-10] and s[i+3] are always addressable. */
static char *slurp(const char *path, long *len, long limit)
{
	int fd = open(path, O_RDONLY);
	if (fd < 0) return NULL;
	struct stat st;
	if (fstat(fd, &st) != 0) { close(fd); return NULL; }
	long size = (long)st.st_size;
	if (limit > 0 && size > limit) size = limit;
	char *buf = malloc((size_t)size + 32);
	if (!buf) { close(fd); return NULL; }
	memset(buf, ' ', 16);
	long got = 0;
	while (got < size) {
		ssize_t r = read(fd, buf + 16 + got, (size_t)(size - got));
		if (r <= 0) break;
		got += r;
	}
	close(fd);
	memset(buf + 16 + got, 0, 16);
	*len = got;
	return buf;
}

/* Token scan shared by both readers: every 'e' marks a number; '\n' starts a new row (the
 * reference's m/n bookkeeping, fun_save_to_file.c:95-108); the scan stops at the wanted count.
 * The text is cut into `C` chunks that start at line starts; a first pass counts each chunk's
 * tokens and line breaks, so every token's ordinal and row are known and the chunks are parsed
 * in parallel, with the checks and values of the sequential scan.  A row with more than `cols`
 * numbers writes into the next row's slots, where the sequential scan lets the later value win:
 * if any row does that, the caller scans again with one chunk (DGH_RESCAN). */
#define DGH_RESCAN (-1000)
static long scan_tokens(const char *s, long len, long rows, long cols, double *outd, long *outl, int C)
{
	const long want = rows * cols;
	pow10_table t;
	pow10_fill(&t);
	long *cut = malloc(sizeof(long) * (size_t)(3 * C + 3));
	if (!cut) return DGH_ERR_NOMEM;
	long *tok0 = cut + C + 1, *row0 = tok0 + C + 1;
	for (int c = 0; c <= C; c++) {
		long at = len * c / C;
		while (c > 0 && c < C && at < len && s[at - 1] != '\n') at++;
		cut[c] = at;
	}
	tok0[0] = row0[0] = 0;
#pragma omp parallel for schedule(static)
	for (int c = 0; c < C; c++) {
		long ne = 0, nl = 0;
		for (long i = cut[c]; i < cut[c + 1]; i++) {
			ne += s[i] == 'e';
			nl += s[i] == '\n';
		}
		tok0[c + 1] = ne;
		row0[c + 1] = nl;
	}
	for (int c = 0; c < C; c++) {
		tok0[c + 1] += tok0[c];
		row0[c + 1] += row0[c];
	}
	int bad = 0, spill = 0;
#pragma omp parallel for schedule(static) reduction(| : bad, spill)
	for (int c = 0; c < C; c++) {
		long num = tok0[c], m = row0[c], n = 0;
		for (long i = cut[c]; i < cut[c + 1] && num < want && !bad; i++) {
			if (s[i] == 'e') {
				const long at = m * cols + n;
				if (i + 3 >= len || i < 9 || s[i - 8] != '.' || at >= want) {
					bad = 1;
					break;
				}
				spill |= n >= cols;
				if (outd) outd[at] = parse_e7(s, i, &t);
				else outl[at] = parse_int_e7(s, i, &t);
				n++;
				num++;
			}
			if (s[i] == '\n') { m++; n = 0; }
		}
	}
	const long total = tok0[C];
	free(cut);
	if (spill && C > 1) return DGH_RESCAN;
	if (bad) return DGH_ERR_FORMAT;
	return total >= want ? want : DGH_ERR_FORMAT;
}

static long read_tokens(const char *path, long rows, long cols, double *outd, long *outl)
{
	if (!path || rows <= 0 || cols <= 0 || (!outd && !outl)) return DGH_ERR_ARG;
	long len;
	char *buf = NULL;
	if (rows * cols == 1) {
		/* a header value: the first line is enough, unless the first number runs past it */
		buf = slurp(path, &len, 4096);
		if (!buf) return DGH_ERR_IO;
		const char *e = memchr(buf + 16, 'e', (size_t)len);
		if (len == 4096 && (!e || e - (buf + 16) + 3 >= len)) {
			free(buf);
			buf = NULL;
		}
	}
	if (!buf) buf = slurp(path, &len, 0);
	if (!buf) return DGH_ERR_IO;
	long r = scan_tokens(buf + 16, len, rows, cols, outd, outl, len < (1L << 20) ? 1 : 4 * omp_get_max_threads());
	if (r == DGH_RESCAN) r = scan_tokens(buf + 16, len, rows, cols, outd, outl, 1);
	free(buf);
	return r;
}

long dgh_read_matrix(const char *path, double *out, long rows, long cols)
{
	return read_tokens(path, rows, cols, out, NULL);
}

long dgh_read_int_matrix(const char *path, long *out, long rows, long cols)
{
	return read_tokens(path, rows, cols, NULL, out);
}

/* Calculate_Tri / Calculate_Point_Num / Mesh_Input (fun_DG.c:70-119) */
int dgh_read_mesh(const char *prefix, dgh_mesh *mo)
{
	if (!prefix || !mo) return DGH_ERR_ARG;
	memset(mo, 0, sizeof *mo);
	char pe[4096], pn[4096], pb[4096];
	snprintf(pe, sizeof pe, "%s.ele", prefix);
	snprintf(pn, sizeof pn, "%s.node", prefix);
	snprintf(pb, sizeof pb, "%s.neigh", prefix);
	long K, P;
	long r = dgh_read_int_matrix(pe, &K, 1, 1);
	if (r < 0) return (int)r;
	r = dgh_read_int_matrix(pn, &P, 1, 1);
	if (r < 0) return (int)r;
	if (K <= 0 || P <= 0) return DGH_ERR_FORMAT;
	long *tri = malloc(sizeof(long) * (K + 1) * 5);
	long *nb = malloc(sizeof(long) * (K + 1) * 4);
	double *pt = malloc(sizeof(double) * (P + 1) * 4);
	mo->Point = malloc(sizeof(double) * P * 2);
	mo->Triangle = malloc(sizeof(long) * K * 3);
	mo->neighbor = malloc(sizeof(long) * K * 3);
	mo->attribute = malloc(sizeof(long) * K);
	int rc = DGH_OK;
	if (!tri || !nb || !pt || !mo->Point || !mo->Triangle || !mo->neighbor || !mo->attribute) { rc = DGH_ERR_NOMEM; goto done; }
	if ((r = dgh_read_int_matrix(pe, tri, K + 1, 5)) < 0) { rc = (int)r; goto done; }
	if ((r = dgh_read_int_matrix(pb, nb, K + 1, 4)) < 0) { rc = (int)r; goto done; }
	if ((r = dgh_read_matrix(pn, pt, P + 1, 4)) < 0) { rc = (int)r; goto done; }
	for (long i = 0; i < K; i++) {
		for (int j = 1; j <= 3; j++) {
			mo->Triangle[i * 3 + j - 1] = tri[(i + 1) * 5 + j];
			mo->neighbor[i * 3 + j - 1] = nb[(i + 1) * 4 + j];
		}
		mo->attribute[i] = tri[(i + 1) * 5 + 4];
	}
	for (long i = 0; i < P; i++) {
		mo->Point[i * 2 + 0] = pt[(i + 1) * 4 + 1];
		mo->Point[i * 2 + 1] = pt[(i + 1) * 4 + 2];
	}
	mo->K = K;
	mo->n_points = P;
done:
	free(tri);
	free(nb);
	free(pt);
	if (rc != DGH_OK) dgh_free_mesh(mo);
	return rc;
}

void dgh_free_mesh(dgh_mesh *m)
{
	if (!m) return;
	free(m->Point);
	free(m->Triangle);
	free(m->neighbor);
	free(m->attribute);
	memset(m, 0, sizeof *m);
}

/* ---------------------------------------------------------------- geometry -------------- */

typedef struct { double x[3], z[3]; } tri_xy;

static inline tri_xy corners(const dgh_setup_in *in, long e)
{
	tri_xy t;
	for (int v = 0; v < 3; v++) {
		long p = in->Triangle[e * 3 + v] - 1;
		t.x[v] = in->Point[p * 2 + 0];
		t.z[v] = in->Point[p * 2 + 1];
	}
	return t;
}

/* EdgeLength (fun_DG.c:122-144): edge 0 = v0v1, 1 = v1v2, 2 = v0v2 */
static inline void edge_lengths(const tri_xy *t, double L[3])
{
	L[0] = sqrt(pow(t->x[0] - t->x[1], 2) + pow(t->z[0] - t->z[1], 2));
	L[1] = sqrt(pow(t->x[1] - t->x[2], 2) + pow(t->z[1] - t->z[2], 2));
	L[2] = sqrt(pow(t->x[0] - t->x[2], 2) + pow(t->z[0] - t->z[2], 2));
}

/* Normals via the incircle tangency points (fun_DG.c:456-554) */
static void outward_normals(const tri_xy *t, const double L[3], double n[3][2])
{
	double ang[3];
	ang[0] = acos((L[0] * L[0] + L[2] * L[2] - L[1] * L[1]) / (2 * L[0] * L[2]));
	ang[1] = acos((L[0] * L[0] + L[1] * L[1] - L[2] * L[2]) / (2 * L[0] * L[1]));
	ang[2] = acos((L[1] * L[1] + L[2] * L[2] - L[0] * L[0]) / (2 * L[1] * L[2]));
	double inc[2];
	double px[3][2] = {{t->x[0], t->z[0]}, {t->x[1], t->z[1]}, {t->x[2], t->z[2]}};
	for (int j = 0; j < 2; j++)
		inc[j] = (L[1] * px[0][j] + L[2] * px[1][j] + L[0] * px[2][j]) / (L[1] + L[2] + L[0]);
	/* face f runs from corner a to corner b; the tangent length from a is |inc - a| cos(ang_a/2) */
	static const int fa[3] = {0, 1, 2}, fb[3] = {1, 2, 0};
	for (int f = 0; f < 3; f++) {
		int a = fa[f], b = fb[f];
		double tl = sqrt(pow(inc[0] - px[a][0], 2) + pow(inc[1] - px[a][1], 2)) * cos(0.5 * ang[a]);
		double foot[2], d[2];
		for (int j = 0; j < 2; j++) {
			foot[j] = px[a][j] + (tl / L[f]) * (px[b][j] - px[a][j]);
			d[j] = foot[j] - inc[j];
		}
		n[f][0] = (d[0] * 1.0 + d[1] * 0.0) / sqrt(pow(d[0], 2) + pow(d[1], 2));
		n[f][1] = (d[0] * 0.0 + d[1] * 1.0) / sqrt(pow(d[0], 2) + pow(d[1], 2));
	}
}

double dgh_ricker(long step, double dt, double t0, double fp, double pi)
{
	double t = dt * step;
	return (1 - 2 * pi * pi * fp * fp * (t - t0) * (t - t0)) * exp(-pi * pi * fp * fp * (t - t0) * (t - t0));
}

/* Ricker_Delay_Time (fun_DG.c:1289-1310): first step where the rising wavelet is below 1e-8 */
static double ricker_delay(double dt, double fp, double pi)
{
	for (long T = 0;; T++) {
		double t1 = T * dt;
		double s1 = (1 - 2 * pi * pi * fp * fp * (t1) * (t1)) * exp(-pi * pi * fp * fp * (t1) * (t1));
		double t2 = (T + 1) * dt;
		double s2 = (1 - 2 * pi * pi * fp * fp * (t2) * (t2)) * exp(-pi * pi * fp * fp * (t2) * (t2));
		if (s2 > s1 && s2 < 1e-8) return t2 * 2.6;
		if (T > 100000000L) return NAN;
	}
}

/* Rstoxy (fun_DG.c:864-876) for one node */
static inline void node_xy(const tri_xy *t, double r, double s, double *x, double *z)
{
	*x = -(r + s) / 2 * t->x[0] + (r + 1) / 2 * t->x[1] + (s + 1) / 2 * t->x[2];
	*z = -(r + s) / 2 * t->z[0] + (r + 1) / 2 * t->z[1] + (s + 1) / 2 * t->z[2];
}

/* Absorbing_Fun's per-node rules (fun_DG.c:926-1003); later rules overwrite earlier ones */
static double sponge_at(double x, double z, double a, const dgh_setup_in *in)
{
	const double bx = in->bound_x, bz = in->bound_z, mw = in->model_w, mh = in->model_h;
	const double Lx = bx, Lz = bz, beta = in->beta, pi = in->pi;
	double d, dx, dz;
	if (x < bx && (z > bz && z < bz + mh)) { d = bx - x; a = 0.5 + 0.5 * cos(beta * d * pi / Lx); }
	if (x > bx + mw && (z > bz && z < bz + mh)) { d = x - bx - mw; a = 0.5 + 0.5 * cos(beta * d * pi / Lx); }
	if (z < bz && (x > bx && x < bx + mw)) { d = bz - z; a = 0.5 + 0.5 * cos(beta * d * pi / Lz); }
	if (z > bz + mh && (x > bx && x < bx + mw)) { d = z - bz - mh; a = 0.5 + 0.5 * cos(beta * d * pi / Lz); }
	dx = fabs(x - bx);
	dz = fabs(z - bz);
	d = sqrt(dx * dx + dz * dz);
	if (x < bx && z < bz && d < bx) a = 0.5 + 0.5 * cos(beta * d * pi / Lx);
	dx = fabs(x - (bx + mw));
	dz = fabs(z - bz);
	d = sqrt(dx * dx + dz * dz);
	if (x > bx + mw && z < bz && d < bx) a = 0.5 + 0.5 * cos(beta * d * pi / Lx);
	dx = fabs(x - (bx + mw));
	dz = fabs(z - (bz + mh));
	d = sqrt(dx * dx + dz * dz);
	if (x > bx + mw && z > bz + mh && d < bx) a = 0.5 + 0.5 * cos(beta * d * pi / Lx);
	dx = fabs(x - bx);
	dz = fabs(z - (bz + mh));
	d = sqrt(dx * dx + dz * dz);
	if (x < bx && z > bz + mh && d < bx) a = 0.5 + 0.5 * cos(beta * d * pi / Lx);
	return a;
}

static inline int outside_box(double x, double z, const dgh_setup_in *in)
{
	return x > (in->bound_x + in->model_w) || x < in->bound_x || z > (in->bound_z + in->model_h) || z < in->bound_z;
}

/* node number (1-based) of a triangle's corner slot: slot 0 -> 6, 1 -> 1, 2 -> 3 (fun_DG.c:329-340) */
static const long corner_node[3] = {6, 1, 3};

typedef struct { double x; long q; } x_index; /* a query position's x and its index */
static int cmp_by_x(const void *a, const void *b)
{
	const x_index *u = a, *v = b;
	return u->x < v->x ? -1 : (u->x > v->x ? 1 : (u->q < v->q ? -1 : (u->q > v->q)));
}
static int cmp_long_pair(const void *a, const void *b)
{
	const long *x = a, *y = b;
	return x[0] != y[0] ? (x[0] < y[0] ? -1 : 1) : (x[1] < y[1] ? -1 : (x[1] > y[1]));
}

/* For each of n query positions, the 1-based index of the first (last = 0) or last (last = 1)
 * vertex whose coordinates both lie within tol of it, or -1: the matching rule of Get_Source /
 * Get_Receiver, evaluated with one pass over the vertices. */
static void match_vertices(const double *Point, long P, const double *pos, long n, double tol, int last, long *out)
{
	if (n <= 0) return;
	x_index *ord = malloc(sizeof(x_index) * (size_t)n);
	for (long q = 0; q < n; q++) out[q] = -1;
	if (!ord) { /* out of memory: fall back to the direct scan */
		for (long q = 0; q < n; q++)
			for (long i = 0; i < P; i++)
				if (fabs(Point[i * 2] - pos[q * 2]) < tol && fabs(Point[i * 2 + 1] - pos[q * 2 + 1]) < tol) {
					out[q] = i + 1;
					if (!last) break;
				}
		return;
	}
	for (long q = 0; q < n; q++) { ord[q].x = pos[2 * q]; ord[q].q = q; }
	qsort(ord, (size_t)n, sizeof(x_index), cmp_by_x);
	/* vertices in parallel; a match keeps the smallest (first) or largest (last) vertex index */
#pragma omp parallel for schedule(static)
	for (long i = 0; i < P; i++) {
		const double px = Point[i * 2], pz = Point[i * 2 + 1];
		/* queries with x > px - tol - a margin (the exact test below decides) */
		const double lo_x = px - 2 * tol;
		long lo = 0, hi = n;
		while (lo < hi) { const long mid = (lo + hi) / 2; if (ord[mid].x < lo_x) lo = mid + 1; else hi = mid; }
		for (long k = lo; k < n && ord[k].x <= px + 2 * tol; k++) {
			const long q = ord[k].q;
			if (fabs(px - pos[q * 2]) < tol && fabs(pz - pos[q * 2 + 1]) < tol) {
#pragma omp critical(dgh_match)
				if (out[q] < 0 || (last ? i + 1 > out[q] : i + 1 < out[q])) out[q] = i + 1;
			}
		}
	}
	free(ord);
}

int dgh_build(const dgh_setup_in *in, dgh_setup_out *out)
{
	if (!in || !out || in->K <= 0 || in->n_points <= 0 || !in->Point || !in->Triangle || !in->neighbor ||
		!in->vp || !in->vs || !in->rho || !in->V || !in->Vr || !in->Vs || !in->inverV || !in->S1 || !in->S2 ||
		!in->S3 || !in->Fekete || in->n_shots < 0 || in->n_rec < 0 || in->bound_x <= 0 || in->bound_z <= 0)
		return DGH_ERR_ARG;
	const long K = in->K, P = in->n_points;
	int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
	for (long e = 0; e < K; e++) {
		const long *t = in->Triangle + e * 3;
		for (int v = 0; v < 3; v++)
			bad |= t[v] < 1 || t[v] > P;
		bad |= t[0] == t[1] || t[1] == t[2] || t[0] == t[2];
		for (int v = 0; v < 3; v++)
			bad |= in->neighbor[e * 3 + v] != -1 && (in->neighbor[e * 3 + v] < 1 || in->neighbor[e * 3 + v] > K);
	}
	if (bad) return DGH_ERR_MESH;

	/* Jacobian (fun_DG.c:421-453) and Normals */
	double *Jac = out->Jacobi ? out->Jacobi : malloc(sizeof(double) * K);
	double *rin = malloc(sizeof(double) * K); /* inscribed diameter per element */
	if (!Jac || !rin) {
		if (!out->Jacobi) free(Jac);
		free(rin);
		return DGH_ERR_NOMEM;
	}
#pragma omp parallel for schedule(static)
	for (long e = 0; e < K; e++) {
		tri_xy t = corners(in, e);
		double L[3];
		edge_lengths(&t, L);
		double xr = (t.x[1] - t.x[0]) * 0.5, yr = (t.z[1] - t.z[0]) * 0.5;
		double xs = (t.x[2] - t.x[0]) * 0.5, ys = (t.z[2] - t.z[0]) * 0.5;
		Jac[e] = xr * ys - xs * yr;
		if (out->Jacobi_Edge)
			for (int j = 0; j < 3; j++) out->Jacobi_Edge[e * 3 + j] = L[j] / 2;
		if (out->normal1 || out->normal2 || out->normal3 || out->Q) {
			double n[3][2];
			outward_normals(&t, L, n);
			double *dst[3] = {out->normal1, out->normal2, out->normal3};
			for (int f = 0; f < 3; f++)
				if (dst[f]) { dst[f][e * 2 + 0] = n[f][0]; dst[f][e * 2 + 1] = n[f][1]; }
			if (out->Q) {
				/* Elastic_A_B + Central_flux (fun_DG.c:1071-1134), A/B formed inline */
				double Cp = in->vp[e], Cs = in->vs[e], den = in->rho[e];
				double miu = den * Cs * Cs, lambda = den * Cp * Cp - 2 * miu;
				double A[5] = {1 / den, 1 / den, lambda + 2 * miu, lambda, miu};
				double B[5] = {1 / den, 1 / den, lambda, lambda + 2 * miu, miu};
				for (int j = 0; j < 3; j++) {
					double nx = n[j][0], nz = n[j][1], JE = L[j] / 2, J = Jac[e];
					double *q = out->Q + e * 30 + j * 10;
					q[0] = 0.5 * nx * A[0] * JE / J;
					q[1] = 0.5 * nz * B[0] * JE / J;
					q[2] = 0.5 * nz * A[1] * JE / J;
					q[3] = 0.5 * nx * B[1] * JE / J;
					q[4] = 0.5 * nx * A[2] * JE / J;
					q[5] = 0.5 * nz * B[2] * JE / J;
					q[6] = 0.5 * nx * A[3] * JE / J;
					q[7] = 0.5 * nz * B[3] * JE / J;
					q[8] = 0.5 * nz * A[4] * JE / J;
					q[9] = 0.5 * nx * B[4] * JE / J;
				}
			}
		}
		/* InDiameter_Min (fun_DG.c:147-176) */
		double a = L[0], b = L[1], c = L[2];
		double s = 0.5 * (a + b + c);
		double S = sqrt(s * (s - a) * (s - b) * (s - c));
		rin[e] = 2 * S / s;
	}
	double min_r = 0.0;
	for (long e = 0; e < K; e++)
		if (e == 0 || rin[e] < min_r) min_r = rin[e];
	free(rin);

	/* Elastic_A_B (fun_DG.c:1071-1088) with the material formulas of DG_leap_Frog_OpenMP.c:252-253 */
	double vmax = in->vp[0];
	for (long e = 1; e < K; e++)
		if (in->vp[e] > vmax) vmax = in->vp[e];
#pragma omp parallel for schedule(static)
	for (long e = 0; e < K; e++) {
		double Cp = in->vp[e], Cs = in->vs[e], den = in->rho[e];
		double miu = den * Cs * Cs, lambda = den * Cp * Cp - 2 * miu;
		if (out->A) {
			double *A = out->A + e * 5;
			A[0] = 1 / den; A[1] = 1 / den; A[2] = lambda + 2 * miu; A[3] = lambda; A[4] = miu;
		}
		if (out->B) {
			double *B = out->B + e * 5;
			B[0] = 1 / den; B[1] = 1 / den; B[2] = lambda; B[3] = lambda + 2 * miu; B[4] = miu;
		}
		if (out->Vp_used) out->Vp_used[e] = in->vp[e];
	}

	/* Calculate_Time_Step (fun_DG.c:179-199) with N = 2, Ricker_Delay_Time */
	out->dt = min_r / vmax / (2 * 2 + 1) * 0.99;
	out->t0 = ricker_delay(out->dt, in->fp, in->pi);
	if (out->wavelet)
		for (long t = 0; t < in->n_steps; t++) out->wavelet[t] = dgh_ricker(t, out->dt, out->t0, in->fp, in->pi);

	/* Get_Source + source vector (fun_DG.c:284-353; DG_leap_Frog_OpenMP.c:233-246): the first
	 * vertex within 1e-3 and the first triangle holding it.  Get_Receiver (fun_DG.c:356-418):
	 * the last vertex within 1e-2 and the last triangle holding it.  The reference scans all
	 * vertices and triangles per source and receiver (O((S + R) K)); here one pass over the
	 * vertices (binary search among the positions sorted by x) and one over the triangles give
	 * the same indices. */
	int rc = DGH_OK;
	long *src_node = NULL, *rec_node = NULL, *src_tri = NULL, *rec_tri = NULL;
	if (in->n_shots + in->n_rec > 0) {
		const long S = in->n_shots, R = in->n_rec;
		src_node = calloc((size_t)(S + R) * 4, sizeof(long));
		if (!src_node) { rc = DGH_ERR_NOMEM; goto fail; }
		rec_node = src_node + S;
		src_tri = rec_node + R;  /* [S][2] triangle, slot */
		rec_tri = src_tri + 2 * S; /* [R][2] */
		match_vertices(in->Point, P, in->src_pos, S, 1e-3, 0, src_node);
		match_vertices(in->Point, P, in->rec_pos, R, 1e-2, 1, rec_node);
		for (long q = 0; q < 2 * (S + R); q++) src_tri[q] = -1;
		/* vertex -> queries that matched it, as a sorted list of (vertex, query) pairs */
		long nq = 0;
		long *pairs = malloc(sizeof(long) * 2 * (size_t)(S + R));
		if (!pairs) { rc = DGH_ERR_NOMEM; goto fail; }
		for (long q = 0; q < S + R; q++)
			if (src_node[q] > 0) { pairs[2 * nq] = src_node[q]; pairs[2 * nq + 1] = q; nq++; }
		qsort(pairs, (size_t)nq, 2 * sizeof(long), cmp_long_pair);
		/* triangles in parallel; a source keeps the smallest (first) triangle holding its vertex,
		 * a receiver the largest (last) */
#pragma omp parallel for schedule(static)
		for (long e = 0; e < K; e++)
			for (int v = 0; v < 3; v++) {
				const long node = in->Triangle[e * 3 + v];
				long lo = 0, hi = nq;  /* first pair with vertex >= node */
				while (lo < hi) { const long mid = (lo + hi) / 2; if (pairs[2 * mid] < node) lo = mid + 1; else hi = mid; }
				for (long k = lo; k < nq && pairs[2 * k] == node; k++) {
					const long q = pairs[2 * k + 1];
					long *slot = q < S ? src_tri + 2 * q : rec_tri + 2 * (q - S);
#pragma omp critical(dgh_match)
					if (slot[0] < 0 || (q < S ? e + 1 < slot[0] : e + 1 > slot[0])) { slot[0] = e + 1; slot[1] = corner_node[v]; }
				}
			}
		free(pairs);
	}
	for (long m = 0; m < in->n_shots; m++) {
		if (src_node[m] < 0) { rc = DGH_ERR_NOSOURCE; goto fail; }
		const long tri = src_tri[2 * m], local = src_tri[2 * m + 1];
		if (tri < 0) { rc = DGH_ERR_NOSOURCE; goto fail; }
		if (out->source) { out->source[m * 2 + 0] = tri; out->source[m * 2 + 1] = local; }
		if (out->fun) {
			long k = local - 1;
			for (int i = 0; i < NPN; i++) {
				double sum = 0;
				for (int j = 0; j < NPN; j++) sum = sum + in->V[i * 6 + j] * in->V[k * 6 + j];
				out->fun[m * NPN + i] = sum / Jac[tri - 1];
			}
		}
	}

	for (long r = 0; r < in->n_rec; r++) {
		if (rec_node[r] < 0) { rc = DGH_ERR_NORECEIVER; goto fail; }
		const long tri = rec_tri[2 * r], local = rec_tri[2 * r + 1];
		if (tri < 0) { rc = DGH_ERR_NORECEIVER; goto fail; }
		if (out->receiver) { out->receiver[r * 2 + 0] = tri; out->receiver[r * 2 + 1] = local; }
	}
	free(src_node);
	src_node = NULL;

	/* Sponge: Get_Absorb_Square_Num, Get_absorb_square (vertex 0 only), Absorbing_Fun
	 * (fun_DG.c:202-281, 879-1006) */
	{
		long count = 0, filled = 0;
#pragma omp parallel for schedule(static) reduction(+ : count, filled)
		for (long e = 0; e < K; e++) {
			tri_xy t = corners(in, e);
			int any = 0;
			for (int v = 0; v < 3; v++) any |= outside_box(t.x[v], t.z[v], in);
			count += any;
			if (outside_box(t.x[0], t.z[0], in)) {
				filled++;
				if (out->absorb_fun)
					for (int i = 0; i < NPN; i++) {
						double x, z;
						node_xy(&t, in->Fekete[i * 2 + 0], in->Fekete[i * 2 + 1], &x, &z);
						out->absorb_fun[e * NPN + i] = sponge_at(x, z, 1.0, in);
					}
			} else if (out->absorb_fun) {
				for (int i = 0; i < NPN; i++) out->absorb_fun[e * NPN + i] = 1;
			}
		}
		out->absorb_count = count;
		out->absorb_filled = filled;
	}

	/* S assembly (DG_leap_Frog_OpenMP.c:306-314) and IBE (fun_DG.c:1046-1057) */
	if (out->S)
		for (int j = 0; j < NPN; j++)
			for (int n = 0; n < NFN; n++) {
				out->S[0 * 18 + j * 3 + n] = in->S1[j * 3 + n];
				out->S[1 * 18 + j * 3 + n] = in->S2[j * 3 + n];
				out->S[2 * 18 + j * 3 + n] = in->S3[j * 3 + n];
			}
	static const long ibe_p2[9] = {6, 4, 1, 1, 2, 3, 6, 5, 3};
	if (out->ibe) memcpy(out->ibe, ibe_p2, sizeof ibe_p2);

	/* Neighbor_Edge (fun_DG.c:557-739) and NeighborNodes (fun_DG.c:1195-1276).
	 * Own face f joins corners (f, f+1) for f = 0, 1 and (2, 0) for f = 2; the neighbour's
	 * matching edge id is 1 for its {v0,v1}, 2 for {v1,v2}, 3 for {v0,v2}; a face is flipped
	 * relative to the neighbour's when their first vertices (v0 for faces 0 and 2, v1 for
	 * face 1) differ. */
	if (out->Neighbor || out->Edge || out->Edge_flag || out->Node_Neighbor) {
		static const int own_a[3] = {0, 1, 2}, own_b[3] = {1, 2, 0};
		static const int first_of_edge[3] = {0, 1, 0};
#pragma omp parallel for schedule(static)
		for (long e = 0; e < K; e++) {
			const long *T = in->Triangle + e * 3;
			for (int f = 0; f < 3; f++) {
				/* Triangle's neighbour k lies opposite vertex k: face f is opposite vertex (f+2)%3 */
				long nbr = in->neighbor[e * 3 + (f + 2) % 3];
				if (nbr == -1) nbr = 0;
				long edge = 0;
				if (nbr) {
					const long *t = in->Triangle + (nbr - 1) * 3;
					long A = T[own_a[f]], B = T[own_b[f]];
					static const int ea[3] = {0, 1, 0}, eb[3] = {1, 2, 2};
					for (int g = 0; g < 3; g++)
						if ((t[ea[g]] == A && t[eb[g]] == B) || (t[ea[g]] == B && t[eb[g]] == A)) edge = g + 1;
				}
				if (out->Neighbor) out->Neighbor[e * 3 + f] = nbr ? nbr : 1;
				if (out->Edge) out->Edge[e * 3 + f] = edge;
				if (out->Edge_flag) out->Edge_flag[e * 3 + f] = edge ? 1 : 0;
				if (out->Node_Neighbor) {
					long *nn = out->Node_Neighbor + e * 9 + f * 3;
					if (edge) {
						const long *t = in->Triangle + (nbr - 1) * 3;
						long their_first = t[first_of_edge[edge - 1]];
						long my_first = T[f == 2 ? 0 : f];
						const long *ord = ibe_p2 + (edge - 1) * 3;
						for (int i = 0; i < NFN; i++) nn[i] = (my_first == their_first) ? ord[i] : ord[NFN - 1 - i];
					} else {
						nn[0] = nn[1] = nn[2] = 1;
					}
				}
			}
		}
	}

	/* Dx_Dz (fun_DG.c:1137-1192) */
	if (out->Dx || out->Dz) {
#pragma omp parallel for schedule(static)
		for (long e = 0; e < K; e++) {
			tri_xy t = corners(in, e);
			double Xr = (t.x[1] - t.x[0]) * 0.5, Zr = (t.z[1] - t.z[0]) * 0.5;
			double Xs = (t.x[2] - t.x[0]) * 0.5, Zs = (t.z[2] - t.z[0]) * 0.5;
			double J = Xr * Zs - Xs * Zr;
			double Rx = Zs / J, Rz = -Xs / J, Sx = -Zr / J, Sz = Xr / J;
			double dxd[6][6], dzd[6][6];
			for (int i = 0; i < NPN; i++)
				for (int n = 0; n < NPN; n++) {
					dxd[i][n] = Rx * in->Vr[i * 6 + n] + Sx * in->Vs[i * 6 + n];
					dzd[i][n] = Rz * in->Vr[i * 6 + n] + Sz * in->Vs[i * 6 + n];
				}
			for (int p = 0; p < NPN; p++)
				for (int q = 0; q < NPN; q++) {
					double f1 = 0, f2 = 0;
					for (int k = 0; k < NPN; k++) {
						f1 = f1 + dxd[p][k] * in->inverV[k * 6 + q];
						f2 = f2 + dzd[p][k] * in->inverV[k * 6 + q];
					}
					if (out->Dx) out->Dx[e * 36 + p * 6 + q] = f1;
					if (out->Dz) out->Dz[e * 36 + p * 6 + q] = f2;
				}
		}
	}

fail:
	free(src_node);
	if (!out->Jacobi) free(Jac);
	return rc;
}

/* Save_Data / Save_Record (fun_save_to_file.c:233-281) with a status instead of exit(0) */
/* "%0.14f " of v into out (at least 512 bytes), returning the length.  A double is M * 2^E
 * (M < 2^53); M * 10^14 fits in 128 bits, so v * 10^14 is that product shifted right by -E,
 * rounded to nearest with ties to even on the bits shifted out — the correctly rounded decimal
 * that printf writes.  Values with E > 0 (|v| >= 2^53), infinities and NaN go to snprintf; values
 * below 2^-127 * 2^53 round to a signed zero. */
static int format_f14(char *out, double v)
{
	uint64_t bits;
	memcpy(&bits, &v, sizeof bits);
	const int neg = (int)(bits >> 63), ex = (int)((bits >> 52) & 0x7ff);
	const uint64_t man = bits & ((1ULL << 52) - 1);
	if (ex == 0x7ff) return snprintf(out, 512, "%0.14f ", v);
	const uint64_t M = ex ? man | (1ULL << 52) : man;
	const int E = ex ? ex - 1075 : -1074;
	if (E > 0) return snprintf(out, 512, "%0.14f ", v);
	const unsigned __int128 P = (unsigned __int128)M * 100000000000000ULL;  /* < 2^100 */
	const int sh = -E;
	unsigned __int128 q = 0;
	if (sh < 128) {
		q = P >> sh;
		if (sh > 0) {
			const unsigned __int128 rem = P - (q << sh), half = (unsigned __int128)1 << (sh - 1);
			if (rem > half || (rem == half && (q & 1))) q++;
		}
	}
	uint64_t ip, fp;
	if (q >> 64) {
		ip = (uint64_t)(q / 100000000000000ULL);
		fp = (uint64_t)(q % 100000000000000ULL);
	} else {
		const uint64_t q64 = (uint64_t)q;
		ip = q64 / 100000000000000ULL;
		fp = q64 % 100000000000000ULL;
	}
	char *o = out;
	if (neg) *o++ = '-';
	char digits[24];
	int nd = 0;
	do {
		digits[nd++] = (char)('0' + ip % 10);
		ip /= 10;
	} while (ip);
	while (nd) *o++ = digits[--nd];
	*o++ = '.';
	for (int k = 13; k >= 0; k--) {
		o[k] = (char)('0' + fp % 10);
		fp /= 10;
	}
	o += 14;
	*o++ = ' ';
	return (int)(o - out);
}

/* The rows [r0, r1) as Save_Data prints them ("%0.14f " per value, a line break per row), into
 * a growing buffer; 0 on success. */
typedef struct { char *p; size_t len, cap; } text_buf;
static int format_rows(text_buf *b, const double *m, long r0, long r1, long cols)
{
	char tmp[512];
	b->len = 0;
	for (long i = r0; i < r1; i++) {
		for (long j = 0; j <= cols; j++) {
			int n = j < cols ? format_f14(tmp, m[i * cols + j]) : 1;
			if (j == cols) tmp[0] = '\n';
			if (n < 0 || n >= (int)sizeof tmp) return -1;
			if (b->len + (size_t)n > b->cap) {
				size_t cap = 2 * b->cap + (size_t)n + 4096;
				char *q = realloc(b->p, cap);
				if (!q) return -1;
				b->p = q;
				b->cap = cap;
			}
			memcpy(b->p + b->len, tmp, (size_t)n);
			b->len += (size_t)n;
		}
	}
	return 0;
}

int dgh_write_matrix(const char *path, const double *m, long rows, long cols)
{
	if (!path || (!m && rows > 0) || rows < 0 || cols < 1) return DGH_ERR_ARG;
	FILE *fp = fopen(path, "wb");
	if (!fp) return DGH_ERR_IO;
	/* blocks of rows, each split over the threads into private buffers that are then written in
	 * row order: the same bytes as the sequential fprintf loop of Save_Data */
	const int T = omp_get_max_threads();
	text_buf *bufs = calloc((size_t)T, sizeof(text_buf));
	int rc = bufs ? DGH_OK : DGH_ERR_NOMEM;
	const long block = 8192L * T;
	for (long r0 = 0; r0 < rows && rc == DGH_OK; r0 += block) {
		const long r1 = r0 + block < rows ? r0 + block : rows;
		int bad = 0;
#pragma omp parallel num_threads(T) reduction(| : bad)
		{
			const int k = omp_get_thread_num(), n = omp_get_num_threads();
			const long a = r0 + (r1 - r0) * k / n, z = r0 + (r1 - r0) * (k + 1) / n;
			bufs[k].len = 0;
			bad |= format_rows(&bufs[k], m, a, z, cols) != 0;
		}
		if (bad) rc = DGH_ERR_NOMEM;
		for (int k = 0; k < T && rc == DGH_OK; k++)
			if (bufs[k].len && fwrite(bufs[k].p, 1, bufs[k].len, fp) != bufs[k].len) rc = DGH_ERR_IO;
	}
	if (bufs)
		for (int k = 0; k < T; k++) free(bufs[k].p);
	free(bufs);
	if (fclose(fp) != 0 && rc == DGH_OK) rc = DGH_ERR_IO;
	return rc;
}

int dgh_write_binary(const char *path, const double *m, long n)
{
	if (!path || (!m && n > 0) || n < 0) return DGH_ERR_ARG;
	FILE *fp = fopen(path, "wb");
	if (!fp) return DGH_ERR_IO;
	int rc = (n == 0 || fwrite(m, sizeof(double), (size_t)n, fp) == (size_t)n) ? DGH_OK : DGH_ERR_IO;
	if (fclose(fp) != 0 && rc == DGH_OK) rc = DGH_ERR_IO;
	return rc;
}

int dgh_write_record(const char *path, const double *m, long rows)
{
	return dgh_write_matrix(path, m, rows, 1);
}
