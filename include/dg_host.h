/*
 * dg_host.h — host-side set-up for the DG time loop (plain C, no GPU).
 *
 * Produces, from a triangle mesh and a medium, every array the per-step kernels read, with the
 * same values the reference's own host code computes (bit-for-bit when compiled without FP
 * contraction, as the reference must be).  It mirrors, function by function:
 *   dgh_read_matrix        ReadDouble                    fun_save_to_file.c:22-113
 *   dgh_read_int_matrix    ReadInt                       fun_save_to_file.c:116-204
 *   dgh_read_mesh          Calculate_Tri/_Point_Num,
 *                          Mesh_Input                    fun_DG.c:70-119
 *   dgh_build              Normals, Jacobian, Get_Source, Get_Receiver, source vector,
 *                          Calculate_Time_Step, Ricker_Delay_Time, Get_absorb_square,
 *                          Absorbing_Fun, Elastic_A_B, S assembly, Neighbor_Edge, IBE,
 *                          NeighborNodes, Dx_Dz, Central_flux, Ricker_Source table
 *                          (fun_DG.c:122-1310; DG_leap_Frog_OpenMP.c:203-356)
 *   dgh_write_matrix       Save_Data ("%0.14f ")         fun_save_to_file.c:233-255
 *   dgh_write_record       Save_Record                   fun_save_to_file.c:260-281
 *   dgh_write_binary       (new) the same values as raw little-endian doubles
 * Differences from the reference, all deliberate: no 100 MB input cap (fun_save_to_file.c:36);
 * every function returns a status instead of printing and carrying on or calling exit();
 * the absorbing list is used with its filled length; receivers are stored with stride 2.
 * All index arrays are 1-based `long` (int64), exactly as the reference produces them.
 */
#ifndef DG_HOST_H
#define DG_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

#define DGH_OK 0
#define DGH_ERR_IO -1          /* file missing or unreadable */
#define DGH_ERR_FORMAT -2      /* file holds fewer values than asked, or a malformed number */
#define DGH_ERR_ARG -3         /* null pointer / non-positive size */
#define DGH_ERR_NOSOURCE -4    /* a source position is not within 1e-3 of a mesh vertex */
#define DGH_ERR_NORECEIVER -5  /* a receiver position is not within 1e-2 of a mesh vertex */
#define DGH_ERR_MESH -6        /* vertex index out of range or degenerate triangle */
#define DGH_ERR_NOMEM -7

/* Value-for-value restatement of the reference parser on one "%16.7e" token whose 'e' sits at
 * s[i] (the digits are at s[i-9..i-1], the sign at s[i-10]); exposed for tests. */
double dgh_parse_e7(const char *s, long i);

/* Round each value through the "%16.7e" text format and the reference parser, i.e. give the
 * value a mesh coordinate has after the text round trip of the reference pipeline. */
void dgh_quantize_e7(double *x, long n);

/* Parse `rows x cols` numbers from a MATLAB -ascii file.  Returns the number of values read
 * (>= 0, == rows*cols on success) or a negative DGH_ERR_*. */
long dgh_read_matrix(const char *path, double *out, long rows, long cols);
long dgh_read_int_matrix(const char *path, long *out, long rows, long cols);

typedef struct {
	long K;          /* triangles */
	long n_points;   /* vertices */
	double *Point;   /* [n_points][2] x, z */
	long *Triangle;  /* [K][3] 1-based vertex ids */
	long *neighbor;  /* [K][3] 1-based neighbour opposite vertex k, -1 none (Triangle's .neigh) */
	long *attribute; /* [K] region attribute */
} dgh_mesh;

/* Read prefix.ele / prefix.node / prefix.neigh (converted Triangle format).  Allocates the
 * arrays of *m; release with dgh_free_mesh. */
int dgh_read_mesh(const char *prefix, dgh_mesh *m);
void dgh_free_mesh(dgh_mesh *m);

typedef struct {
	/* mesh */
	long K, n_points;
	const double *Point;     /* [n_points][2] */
	const long *Triangle;    /* [K][3] 1-based */
	const long *neighbor;    /* [K][3] 1-based, -1 none (opposite-vertex convention) */
	/* medium, per element: vp, vs, rho -> Lambda, Miu, Den (DG_leap_Frog_OpenMP.c:249-278) */
	const double *vp, *vs, *rho;
	/* operator matrices as read from the text files */
	const double *V;         /* [6][6] */
	const double *Vr, *Vs;   /* [6][6] */
	const double *inverV;    /* [6][6] */
	const double *S1, *S2, *S3; /* [6][3] each */
	const double *Fekete;    /* [6][2] reference-element nodes */
	/* compile-time knobs of the reference (dg.h), here run-time */
	double fp;               /* Ricker peak frequency (Fp) */
	double pi;               /* value of Pi (the reference uses 3.1415) */
	double beta;             /* sponge strength (0.1) */
	double bound_x, bound_z, model_w, model_h;
	/* sources (one per shot) and receivers: positions that must coincide with vertices */
	long n_shots;
	const double *src_pos;   /* [n_shots][2] */
	long n_rec;
	const double *rec_pos;   /* [n_rec][2] */
	long n_steps;            /* length of the wavelet table */
} dgh_setup_in;

/* Caller-allocated outputs; any pointer may be NULL to skip that array (Dx/Dz/Q/normals are
 * only needed by the bit-exact reference-operator path). */
typedef struct {
	double dt, t0;           /* Calculate_Time_Step, Ricker_Delay_Time */
	long absorb_count;       /* Get_Absorb_Square_Num */
	long absorb_filled;      /* entries Get_absorb_square actually lists */
	double *A, *B;           /* [K][5] */
	double *Jacobi;          /* [K] */
	double *Jacobi_Edge;     /* [K][3] */
	double *normal1, *normal2, *normal3; /* [K][2] */
	double *Q;               /* [K][3][5][2] */
	double *Dx, *Dz;         /* [K][6][6] */
	double *S;               /* [3][6][3] */
	long *ibe;               /* [3][3] */
	long *Neighbor;          /* [K][3] edge-ordered, 1-based, boundary -> 1 */
	long *Edge;              /* [K][3] neighbour's matching edge 1..3, 0 none */
	long *Edge_flag;         /* [K][3] */
	long *Node_Neighbor;     /* [K][3][3] 1-based neighbour node per face node */
	double *absorb_fun;      /* [K][6] */
	long *source;            /* [n_shots][2] (triangle, node) 1-based */
	double *fun;             /* [n_shots][6] */
	long *receiver;          /* [n_rec][2] (triangle, node) 1-based, stride 2 */
	double *wavelet;         /* [n_steps] Ricker_Source(t, dt, t0) */
	double *Vp_used;         /* [K] (optional copy of vp) */
} dgh_setup_out;

int dgh_build(const dgh_setup_in *in, dgh_setup_out *out);

/* The per-step source amplitude, Ricker_Source (fun_DG.c:1279-1286). */
double dgh_ricker(long step, double dt, double t0, double fp, double pi);

/* Text writers of fun_save_to_file.c: "%0.14f " per value, one row per line.  Rows are formatted
 * on OpenMP threads and written in order, so the file holds the bytes of the sequential loop. */
int dgh_write_matrix(const char *path, const double *m, long rows, long cols);
int dgh_write_record(const char *path, const double *m, long rows);
/* n doubles as raw bytes (a snapshot or trace dump that reads back exactly). */
int dgh_write_binary(const char *path, const double *m, long n);

const char *dgh_strerror(int code);

#ifdef __cplusplus
}
#endif
#endif
