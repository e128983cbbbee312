/*
 * CPU oracle for the pybrown_b200 parity tests.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C99, single-threaded, FP64
 * restatement of pyBrown's native hydrodynamics (src/bdsim/clib/diff_tensor.c
 * and src/bdsim/clib/bead.c).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker.  The
 * product (pybrown_b200) never links it and has no CPU fallback.
 *
 * It exports the reference's own symbol names and signatures so that the
 * reference's unittest suites can be pointed at it (oracle/run_reference_suite.py)
 * -- that is how this restatement is pinned against every known-answer value
 * the reference's tests hold (HYDROLIB, BD_BOX, the pure-Python restatement,
 * the permutation-symmetry and the trajectory tests).
 *
 * Numerics follow the reference operation by operation where the order of
 * floating-point additions matters (image loops in L1-ball order, real-space
 * sum before reciprocal sum, m-series in increasing m).  The one deliberate
 * difference: the 6x6 two-bead RPY mobility is inverted with an in-house
 * Gauss-Jordan elimination with partial pivoting instead of LAPACK
 * dgetrf_/dgetri_ (diff_tensor.c:1629-1641), so the oracle needs no LAPACK.
 */

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------- */
/* Periodic geometry (bead.c)                                                */
/* ------------------------------------------------------------------------- */

/* Minimum-image shift with the reference's while-loop semantics
 * (bead.c:44-73): first pull down while x >= L/2, then push up while
 * x <= -L/2.  The result lies in (-L/2, L/2]. */
static double orc_min_image(double x, double L)
{
	while (x >= L / 2.0) x -= L;
	while (x <= -L / 2.0) x += L;
	return x;
}

/* bead.c:27-95.  pointers[(j*N + i)*3 + c] = minimg(r_i - r_j)_c for i > j and
 * the negated vector at [(i*N + j)*3 + c].  The diagonal is left untouched. */
void pointer_pbc_matrix(double *positions, int number_of_beads, double box_length, double *pointers)
{
	int N = number_of_beads;
	for (int j = 0; j < N; j++) {
		for (int i = j + 1; i < N; i++) {
			double d[3];
			for (int c = 0; c < 3; c++)
				d[c] = orc_min_image(positions[3 * i + c] - positions[3 * j + c], box_length);
			for (int c = 0; c < 3; c++) {
				pointers[3 * i + 3 * j * N + c] = d[c];
				pointers[3 * j + 3 * i * N + c] = -d[c];
			}
		}
	}
}

/* bead.c:99-158 (immobile beads; kept for ABI completeness). */
void pointer_immobile_pbc_matrix(double *positions_mobile, double *positions_immobile,
                                 int number_of_mobile, int number_of_immobile,
                                 double box_length, double *pointers)
{
	for (int j = 0; j < number_of_immobile; j++)
		for (int i = 0; i < number_of_mobile; i++)
			for (int c = 0; c < 3; c++)
				pointers[3 * j + 3 * i * number_of_immobile + c] =
					orc_min_image(positions_immobile[3 * j + c] - positions_mobile[3 * i + c], box_length);
}

/* bead.c:169-218 plus overlap_pbc/distance_pbc (:222-260).  The per-axis
 * pre-filter is part of the semantics: a pair whose raw separation along one
 * axis lies strictly between the radii sum and L minus the radii sum is never
 * tested, whatever the threshold. */
int check_overlaps(double *positions, double *as, int number_of_beads, double box_length,
                   double overlap_treshold, int *connection_matrix)
{
	int N = number_of_beads;
	for (int j = 0; j < N; j++) {
		for (int i = j + 1; i < N; i++) {
			if (connection_matrix[j + N * i]) continue;
			double r[3];
			for (int c = 0; c < 3; c++) r[c] = positions[3 * i + c] - positions[3 * j + c];
			double rs = as[i] + as[j];
			double rs_pbc = box_length - rs;
			int separated = 0;
			for (int c = 0; c < 3 && !separated; c++)
				separated = ((r[c] > rs) && (r[c] < rs_pbc)) || ((r[c] < -rs) && (r[c] > -rs_pbc));
			if (separated) continue;
			double x = orc_min_image(r[0], box_length);
			double y = orc_min_image(r[1], box_length);
			double z = orc_min_image(r[2], box_length);
			if (sqrt(x * x + y * y + z * z) <= as[i] + as[j] + overlap_treshold) return 1;
		}
	}
	return 0;
}

/* ------------------------------------------------------------------------- */
/* Packed storage helpers (diff_tensor.c:1645-1650)                          */
/* ------------------------------------------------------------------------- */

/* Index of pair (i, j), i >= j, in a column-packed lower triangle of order n. */
static int orc_packed(int i, int j, int n) { return i + j * n - j * (j + 1) / 2; }

/* Pair vector handed in by the Python wrappers: 3 doubles per pair (i > j),
 * j-major upper-triangle order, value r_j - r_i (diffusion.py:40,70). */
static const double *orc_pair_vec(const double *pointers, int i, int j, int N)
{
	return pointers + 3 * orc_packed(i - 1, j, N - 1);
}

/* Scatter a symmetric 3x3 block given as (xx, yy, zz, xy, xz, yz) into
 * blocks (I,J) and (J,I) of the 3N x 3N matrix stored as M[row + col*n3]. */
static void orc_put_block(double *M, int n3, int I, int J, const double b[6], int accumulate)
{
	static const int ra[9] = {0, 1, 2, 1, 0, 2, 0, 2, 1};
	static const int cb[9] = {0, 1, 2, 0, 1, 0, 2, 1, 2};
	static const int comp[9] = {0, 1, 2, 3, 3, 4, 4, 5, 5};
	for (int t = 0; t < 9; t++) {
		long p = (long)(I + ra[t]) + (long)(J + cb[t]) * n3;
		long q = (long)(J + cb[t]) + (long)(I + ra[t]) * n3;
		if (accumulate) {
			M[p] += b[comp[t]];
			if (I != J) M[q] += b[comp[t]];
		} else {
			M[p] = b[comp[t]];
			M[q] = b[comp[t]];
		}
	}
}

/* ------------------------------------------------------------------------- */
/* Free-space RPY (diff_tensor.c:73-166, :483-549)                           */
/* ------------------------------------------------------------------------- */

/* diff_tensor.c:490-549: the three distance regimes of the RPY pair block. */
static void orc_rpy_pair(double ai, double aj, double rx, double ry, double rz, double out[6])
{
	double al = ai > aj ? ai : aj;
	double asm_ = ai > aj ? aj : ai;
	double d2 = rx * rx + ry * ry + rz * rz;
	double d = sqrt(d2);
	double aij2 = ai * ai + aj * aj;
	double r[3] = {rx, ry, rz};
	memset(out, 0, 6 * sizeof(double));
	if (d > ai + aj) {
		double c1 = 1.0 / (8 * ORC_PI * d);
		double c2 = 1.0 + aij2 / (3 * d2);
		double c3 = (1.0 - aij2 / d2) / d2;
		for (int c = 0; c < 3; c++) out[c] = c1 * (c2 + c3 * r[c] * r[c]);
		out[3] = c1 * c3 * rx * ry;
		out[4] = c1 * c3 * rx * rz;
		out[5] = c1 * c3 * ry * rz;
	} else if (d <= al - asm_) {
		double t = 1.0 / (6 * ORC_PI * al);
		out[0] = out[1] = out[2] = t;
	} else {
		double d3 = d2 * d;
		double c1 = 1.0 / (6 * ORC_PI * ai * aj);
		double c2 = 16 * d3 * (ai + aj);
		double c3 = (ai - aj) * (ai - aj) + 3 * d2;
		c3 *= c3;
		double c4 = (c2 - c3) / 32 / d3;
		double c5 = ((ai - aj) * (ai - aj) - d2);
		c5 *= 3 * c5;
		double c6 = c5 / (32 * d3) / d2;
		for (int c = 0; c < 3; c++) out[c] = c1 * (c4 + c6 * r[c] * r[c]);
		out[3] = c1 * c6 * rx * ry;
		out[4] = c1 * c6 * rx * rz;
		out[5] = c1 * c6 * ry * rz;
	}
}

/* diff_tensor.c:73-166. */
void RPY_M_matrix(double *as, double *pointers, int number_of_beads, double *M_matrix)
{
	int N = number_of_beads, n3 = 3 * N;
#pragma omp parallel for schedule(dynamic, 8)
	for (int j = 0; j < N; j++) {
		double self = 1.0 / (6 * ORC_PI * as[j]);
		M_matrix[3 * j + 3 * j * n3] = self;
		M_matrix[3 * j + 1 + (3 * j + 1) * n3] = self;
		M_matrix[3 * j + 2 + (3 * j + 2) * n3] = self;
		for (int i = j + 1; i < N; i++) {
			const double *p = orc_pair_vec(pointers, i, j, N);
			double b[6];
			orc_rpy_pair(as[i], as[j], p[0], p[1], p[2], b);
			orc_put_block(M_matrix, n3, 3 * i, 3 * j, b, 0);
		}
	}
}

/* ------------------------------------------------------------------------- */
/* Smith's Ewald summation of the RPY tensor (diff_tensor.c:170-266, 553-1087) */
/* ------------------------------------------------------------------------- */

/* Visit every integer vector with |x|+|y|+|z| <= kmax in the reference's loop
 * order (x outer, z inner; diff_tensor.c:675-683). */
#define ORC_L1_BALL(kmax, X, Y, Z)                                  \
	for (int X = -(kmax); X <= (kmax); X++)                          \
		for (int Y = -((kmax) - abs(X)); Y <= (kmax) - abs(X); Y++)    \
			for (int Z = -((kmax) - abs(X) - abs(Y)); Z <= (kmax) - abs(X) - abs(Y); Z++)

/* O (Oseen-like) and Q (dipole-like) kernels, diff_tensor.c:1043-1087. */
static void orc_O(double x, double y, double z, double o[6])
{
	double d2 = x * x + y * y + z * z, d = sqrt(d2), d3 = d2 * d;
	o[0] = (1 + x * x / d2) / d;
	o[1] = (1 + y * y / d2) / d;
	o[2] = (1 + z * z / d2) / d;
	o[3] = x * y / d3;
	o[4] = x * z / d3;
	o[5] = y * z / d3;
}

static void orc_Q(double x, double y, double z, double q[6])
{
	double d2 = x * x + y * y + z * z, d = sqrt(d2), d3 = d2 * d, d5 = d3 * d2;
	q[0] = (1 - 3 * x * x / d2) / d3;
	q[1] = (1 - 3 * y * y / d2) / d3;
	q[2] = (1 - 3 * z * z / d2) / d3;
	q[3] = -3 * x * y / d5;
	q[4] = -3 * x * z / d5;
	q[5] = -3 * y * z / d5;
}

static void orc_outer6(double x, double y, double z, double v[6])
{
	v[0] = x * x; v[1] = y * y; v[2] = z * z; v[3] = x * y; v[4] = x * z; v[5] = y * z;
}

/* Self sums O_self and Q_self (diff_tensor.c:652-849). */
static void orc_smith_self(double a, double L, double alpha, int m_max, int n_max, double O[6], double Q[6])
{
	double sqrt_pi = sqrt(ORC_PI), alpha2 = alpha * alpha, alpha3 = alpha * alpha2;
	double o[6], q[6], mm[6];
	memset(O, 0, 6 * sizeof(double));
	memset(Q, 0, 6 * sizeof(double));
	/* O: real space (m != 0) then reciprocal (n != 0) then self term. */
	double o_real = 2 * alpha / sqrt_pi;
	double kexp = -ORC_PI * ORC_PI / alpha2;
	ORC_L1_BALL(m_max, mx, my, mz) {
		if (mx == 0 && my == 0 && mz == 0) continue;
		double ml2 = mx * mx + my * my + mz * mz, ml = sqrt(ml2);
		orc_O(mx, my, mz, o);
		double w = erfc(alpha * ml);
		for (int c = 0; c < 6; c++) O[c] += w * o[c];
		w = o_real * exp(-alpha2 * ml2) / ml2;
		orc_outer6(mx, my, mz, mm);
		for (int c = 0; c < 6; c++) O[c] += w * mm[c];
	}
	double o_rec = 2.0 / ORC_PI;
	ORC_L1_BALL(n_max, nx, ny, nz) {
		if (nx == 0 && ny == 0 && nz == 0) continue;
		double nl2 = nx * nx + ny * ny + nz * nz;
		double w = o_rec / nl2 * exp(kexp * nl2);
		double t = 1.0 / nl2 - kexp;
		orc_outer6(nx, ny, nz, mm);
		for (int c = 0; c < 3; c++) O[c] += w * (1.0 - t * mm[c]);
		for (int c = 3; c < 6; c++) O[c] += w * (-t * mm[c]);
	}
	double s = 1.5 * alpha * a / (sqrt_pi * L);
	for (int c = 0; c < 3; c++) O[c] -= s;

	/* Q: real space (m != 0) then reciprocal then self term. */
	double q_t1 = 2 / sqrt_pi, q_t2 = 2 * alpha3;
	ORC_L1_BALL(m_max, mx, my, mz) {
		if (mx == 0 && my == 0 && mz == 0) continue;
		double ml2 = mx * mx + my * my + mz * mz;
		double am = alpha * sqrt(ml2), am2 = am * am, e = exp(-am2);
		orc_Q(mx, my, mz, q);
		double w = erfc(am) + q_t1 * am * e;
		for (int c = 0; c < 6; c++) Q[c] += w * q[c];
		w = q_t1 * q_t2 * e / ml2;
		orc_outer6(mx, my, mz, mm);
		for (int c = 0; c < 6; c++) Q[c] -= w * mm[c];
	}
	double q_rec = 4 * ORC_PI;
	ORC_L1_BALL(n_max, nx, ny, nz) {
		if (nx == 0 && ny == 0 && nz == 0) continue;
		double nl2 = nx * nx + ny * ny + nz * nz;
		double w = q_rec * exp(kexp * nl2) / nl2;
		orc_outer6(nx, ny, nz, mm);
		for (int c = 0; c < 6; c++) Q[c] += w * mm[c];
	}
	double a3 = a * a * a, L3 = L * L * L;
	s = alpha3 * a3 / (L3 * 3.0 * sqrt_pi);
	for (int c = 0; c < 3; c++) Q[c] -= s;
}

/* Pair sums O(sigma) and Q(sigma), sigma = r / L (diff_tensor.c:853-1039).
 * Real space includes m = 0; reciprocal excludes n = 0. */
static void orc_smith_pair_sums(double sx, double sy, double sz, double alpha, int m_max, int n_max,
                                double O[6], double Q[6])
{
	double sqrt_pi = sqrt(ORC_PI), alpha2 = alpha * alpha, alpha3 = alpha2 * alpha;
	double o[6], q[6], mm[6];
	memset(O, 0, 6 * sizeof(double));
	memset(Q, 0, 6 * sizeof(double));
	double o_real = 2 * alpha / sqrt_pi;
	ORC_L1_BALL(m_max, mx, my, mz) {
		double x = mx + sx, y = my + sy, z = mz + sz;
		double l2 = x * x + y * y + z * z, l = sqrt(l2);
		double w = erfc(alpha * l);
		orc_O(x, y, z, o);
		for (int c = 0; c < 6; c++) O[c] += w * o[c];
		w = o_real * exp(-alpha2 * l2) / l2;
		orc_outer6(x, y, z, mm);
		for (int c = 0; c < 6; c++) O[c] += w * mm[c];
	}
	double kk = ORC_PI * ORC_PI / alpha2, o_rec = 2.0 / ORC_PI;
	ORC_L1_BALL(n_max, nx, ny, nz) {
		if (nx == 0 && ny == 0 && nz == 0) continue;
		double nl2 = nx * nx + ny * ny + nz * nz;
		double ns = nx * sx + ny * sy + nz * sz;
		double e = kk * nl2;
		double w = o_rec / nl2 * exp(-e) * cos(2 * ORC_PI * ns);
		double t = (1.0 + e) / nl2;
		orc_outer6(nx, ny, nz, mm);
		for (int c = 0; c < 3; c++) O[c] += w * (1.0 - t * mm[c]);
		for (int c = 3; c < 6; c++) O[c] += w * (-t * mm[c]);
	}
	double q_t1 = 2.0 / sqrt_pi, q_t2 = 4 * alpha3 / sqrt_pi;
	ORC_L1_BALL(m_max, mx, my, mz) {
		double x = mx + sx, y = my + sy, z = mz + sz;
		double l2 = x * x + y * y + z * z;
		double al = alpha * sqrt(l2), al2 = al * al, e = exp(-al2);
		double w = erfc(al) + q_t1 * al * e;
		orc_Q(x, y, z, q);
		for (int c = 0; c < 6; c++) Q[c] += w * q[c];
		w = q_t2 * e / l2;
		orc_outer6(x, y, z, mm);
		for (int c = 0; c < 6; c++) Q[c] -= w * mm[c];
	}
	double kexp = -ORC_PI * ORC_PI / alpha2, q_rec = 4 * ORC_PI;
	ORC_L1_BALL(n_max, nx, ny, nz) {
		if (nx == 0 && ny == 0 && nz == 0) continue;
		double nl2 = nx * nx + ny * ny + nz * nz;
		double ns = nx * sx + ny * sy + nz * sz;
		double w = q_rec * exp(kexp * nl2) * cos(2 * ORC_PI * ns) / nl2;
		orc_outer6(nx, ny, nz, mm);
		for (int c = 0; c < 6; c++) Q[c] += w * mm[c];
	}
}

/* diff_tensor.c:553-575: self block. */
static void orc_smith_self_block(double a, double L, double alpha, int m_max, int n_max, double out[6])
{
	double c1 = 1.0 / (6 * ORC_PI * a);
	double c2 = 3 * a / (4 * L);
	double c3 = a * a * a / (2 * L * L * L);
	double O[6], Q[6];
	orc_smith_self(a, L, alpha, m_max, n_max, O, Q);
	for (int c = 0; c < 3; c++) out[c] = c1 * (1.0 + c2 * O[c] + c3 * Q[c]);
	for (int c = 3; c < 6; c++) out[c] = c1 * (c2 * O[c] + c3 * Q[c]);
}

/* diff_tensor.c:579-648: pair block, including the overlap fix that swaps
 * the far-field RPY for the overlapping-regime RPY when r < ai + aj. */
static void orc_smith_pair_block(double ai, double aj, double rx, double ry, double rz, double L,
                                 double alpha, int m_max, int n_max, double out[6])
{
	double d2 = rx * rx + ry * ry + rz * rz;
	double c1 = 1.0 / (6 * ORC_PI * ai);
	double c2 = 3 * ai / (4 * L);
	double c3 = (ai == aj) ? ai * ai * ai / (2 * L * L * L) : ai * (ai * ai + aj * aj) / (4 * L * L * L);
	double O[6], Q[6];
	orc_smith_pair_sums(rx / L, ry / L, rz / L, alpha, m_max, n_max, O, Q);
	for (int c = 0; c < 6; c++) out[c] = c1 * (c2 * O[c] + c3 * Q[c]);
	if (d2 < (ai + aj) * (ai + aj)) {
		double d = sqrt(d2), aij2 = ai * ai + aj * aj, near[6];
		double r[3] = {rx, ry, rz};
		orc_rpy_pair(ai, aj, rx, ry, rz, near);
		for (int c = 0; c < 6; c++) out[c] += near[c];
		double f1 = 1.0 / (8 * ORC_PI * d);
		double f2 = 1.0 + aij2 / (3 * d2);
		double f3 = (1.0 - aij2 / d2) / d2;
		for (int c = 0; c < 3; c++) out[c] -= f1 * (f2 + f3 * r[c] * r[c]);
		out[3] -= f1 * f3 * rx * ry;
		out[4] -= f1 * f3 * rx * rz;
		out[5] -= f1 * f3 * ry * rz;
	}
}

/* diff_tensor.c:170-266. */
void RPY_Smith_M_matrix(double *as, double *pointers, double box_length, double alpha, int m_max,
                        int n_max, int number_of_beads, double *M_matrix)
{
	int N = number_of_beads, n3 = 3 * N;
	/* Every (i, j) writes its own two blocks: the columns j are independent.
	 * With -fopenmp (the _omp build) they run on all host cores; the result
	 * is identical to the serial build. */
#pragma omp parallel for schedule(dynamic, 4)
	for (int j = 0; j < N; j++) {
		double b[6];
		orc_smith_self_block(as[j], box_length, alpha, m_max, n_max, b);
		orc_put_block(M_matrix, n3, 3 * j, 3 * j, b, 0);
		for (int i = j + 1; i < N; i++) {
			const double *p = orc_pair_vec(pointers, i, j, N);
			orc_smith_pair_block(as[i], as[j], p[0], p[1], p[2], box_length, alpha, m_max, n_max, b);
			orc_put_block(M_matrix, n3, 3 * i, 3 * j, b, 0);
		}
	}
}

/* ------------------------------------------------------------------------- */
/* Jeffrey-Onishi two-body resistance (diff_tensor.c:270-342, 1190-1625)      */
/* ------------------------------------------------------------------------- */

/* Coefficients of the JO f_m(l) polynomials, index = power of l
 * (Jeffrey & Onishi, J. Fluid Mech. 139 (1984) 261, as tabulated in
 * diff_tensor.c:1385-1545). */
static const double ORC_XF[12][11] = {
	{1},
	{0, 3},
	{0, 9},
	{0, -4, 27, -4},
	{0, -24, 81, 36},
	{0, 0, 72, 243, 72},
	{0, 16, 108, 281, 648, 144},
	{0, 0, 288, 1620, 1515, 1620, 288},
	{0, 0, 576, 4848, 5409, 4524, 3888, 576},
	{0, 0, 1152, 9072, 14752, 26163, 14752, 9072, 1152},
	{0, 0, 2304, 20736, 42804, 115849, 76176, 39264, 20736, 2304},
	{0, 0, 4608, 46656, 108912, 269100, 319899, 269100, 108912, 46656, 4608},
};
static const double ORC_YF[12][11] = {
	{1},
	{0, 1.5},
	{0, 2.25},
	{0, 2, 3.375, 2},
	{0, 6, 5.0625, 18},
	{0, 0, 31.5, 7.59375, 31.5},
	{0, 4, 54, 19.390625, 81, 72},
	{0, 0, 144, 131.625, 149.0859375, 131.625, 144},
	{0, 0, 279, 532.625, 493.62890625, -14.625, 648, 288},
	{0, 0, 576, 1134, 1888.84375, 1496.443359375, 1888.84375, 1134, 576},
	{0, 0, 1152, 1964.25, 6155.4375, 10301.1650390625, 8452.125, -175.5, 3888, 1152},
	{0, 0, 2304, 7128, 11035.5, 21441.4453125, 46486.24755859375, 21441.4453125, 11035.5, 7128, 2304},
};

/* Sum of coefficient * l^k with explicit powers, terms added in increasing k
 * (the order the reference writes them in). */
static double orc_poly(const double *c, double l)
{
	double s = 0.0, p = 1.0;
	int first = 1;
	for (int k = 0; k < 11; k++) {
		if (c[k] != 0.0) {
			if (first) { s = c[k] * p; first = 0; }
			else s += c[k] * p;
		}
		p *= l;
	}
	return s;
}

static double orc_Xg(double l, int k)
{
	double l2 = l * l, p3 = (1 + l) * (1 + l) * (1 + l);
	if (k == 1) return 2 * l2 / p3;
	if (k == 2) return 0.2 * l * (1 + 7 * l + l2) / p3;
	return 1.0 / 42 * (1 + 18 * l - 29 * l2 + 18 * l2 * l + l2 * l2) / p3;
}

static double orc_Yg(double l, int k)
{
	double l2 = l * l, p3 = (1 + l) * (1 + l) * (1 + l);
	if (k == 2) return 4.0 / 15 * l * (2 + l + 2 * l2) / p3;
	return 2.0 / 375 * (16 - 45 * l + 58 * l2 - 45 * l2 * l + 16 * l2 * l2) / p3;
}

/* diff_tensor.c:1190-1236. */
static double orc_XA11(double s, double l)
{
	double s2 = 1.0 - 4.0 / (s * s), lg = log(s2);
	double g1 = orc_Xg(l, 1), g2 = orc_Xg(l, 2), g3 = orc_Xg(l, 3);
	double v = 0.0;
	v += g1 / s2;
	v -= g2 * lg;
	v -= g3 * s2 * lg;
	v += orc_poly(ORC_XF[0], l) - g1;
	for (int m = 2; m <= 10; m += 2) {
		int m1 = (m == 2) ? -2 : m - 2;
		double w = pow(2 / s, m);
		v += w * (pow(2, -m) * pow(1 + l, -m) * orc_poly(ORC_XF[m], l) - g1);
		v += w * (4.0 / (m * m1) * g3 - 2.0 / m * g2);
	}
	return v;
}

/* diff_tensor.c:1240-1284. */
static double orc_YA11(double s, double l)
{
	double s2 = 1.0 - 4.0 / (s * s), lg = log(s2);
	double g2 = orc_Yg(l, 2), g3 = orc_Yg(l, 3);
	double v = 0.0;
	v -= g2 * lg;
	v -= g3 * s2 * lg;
	v += orc_poly(ORC_YF[0], l);
	for (int m = 2; m <= 10; m += 2) {
		int m1 = (m == 2) ? -2 : m - 2;
		double w = pow(2 / s, m);
		v += w * (pow(2, -m) * pow(1 + l, -m) * orc_poly(ORC_YF[m], l) - 2.0 / m * g2);
		v += w * 4.0 / (m * m1) * g3;
	}
	return v;
}

/* diff_tensor.c:1288-1333 (odd m; m1 = m - 2). */
static double orc_XA12(double s, double l)
{
	double s2 = 1.0 - 4.0 / (s * s), lg = log((s + 2) / (s - 2));
	double g1 = orc_Xg(l, 1), g2 = orc_Xg(l, 2), g3 = orc_Xg(l, 3);
	double v = 0.0;
	v += 2.0 / s * g1 / s2;
	v += g2 * lg;
	v += g3 * s2 * lg + 4 * g3 / s;
	for (int m = 1; m <= 11; m += 2) {
		int m1 = m - 2;
		double w = pow(2 / s, m);
		v += w * (pow(2, -m) * pow(1 + l, -m) * orc_poly(ORC_XF[m], l) - g1);
		v += w * (4.0 / (m * m1) * g3 - 2.0 / m * g2);
	}
	return -v;
}

/* diff_tensor.c:1337-1381 (odd m; m1 = m - 2). */
static double orc_YA12(double s, double l)
{
	double s2 = 1.0 - 4.0 / (s * s), lg = log((s + 2) / (s - 2));
	double g2 = orc_Yg(l, 2), g3 = orc_Yg(l, 3);
	double v = 0.0;
	v += g2 * lg;
	v += g3 * s2 * lg;
	v += 4 * g3 / s;
	for (int m = 1; m <= 11; m += 2) {
		int m1 = m - 2;
		double w = pow(2 / s, m);
		v += w * (pow(2, -m) * pow(1 + l, -m) * orc_poly(ORC_YF[m], l) - 2.0 / m * g2);
		v += w * (4.0 / (m * m1) * g3);
	}
	return -v;
}

/* Longitudinal/transverse scalars -> symmetric 3x3 block X r^r^ + Y (1 - r^r^). */
static void orc_xy_block(double X, double Y, double rx, double ry, double rz, double d2, double out[6])
{
	out[0] = X * rx * rx / d2 + Y * (1 - rx * rx / d2);
	out[1] = X * ry * ry / d2 + Y * (1 - ry * ry / d2);
	out[2] = X * rz * rz / d2 + Y * (1 - rz * rz / d2);
	out[3] = (X - Y) * rx * ry / d2;
	out[4] = (X - Y) * rx * rz / d2;
	out[5] = (X - Y) * ry * rz / d2;
}

/* diff_tensor.c:270-342: 18 components (block 11, block 22, block 12). */
void JO_2B_R_matrix(double ai, double aj, double rx, double ry, double rz, double *R_matrix)
{
	double d2 = rx * rx + ry * ry + rz * rz, d = sqrt(d2);
	double s = 2 * d / (ai + aj), l = aj / ai;
	double xa11 = orc_XA11(s, l), ya11 = orc_YA11(s, l);
	double xa22 = l * orc_XA11(s, 1 / l), ya22 = l * orc_YA11(s, 1 / l);
	double xa12 = orc_XA12(s, l), ya12 = orc_YA12(s, l);
	orc_xy_block(xa11, ya11, rx, ry, rz, d2, R_matrix);
	orc_xy_block(xa22, ya22, rx, ry, rz, d2, R_matrix + 6);
	orc_xy_block(xa12, ya12, rx, ry, rz, d2, R_matrix + 12);
	double mult = 6 * ORC_PI * ai;
	for (int k = 0; k < 18; k++) R_matrix[k] *= mult;
}

/* In-place inverse of a small dense matrix (row-major, order n <= 6) by
 * Gauss-Jordan elimination with partial pivoting. */
static void orc_invert_small(double *A, int n)
{
	double aug[6][12];
	for (int r = 0; r < n; r++)
		for (int c = 0; c < 2 * n; c++)
			aug[r][c] = (c < n) ? A[r * n + c] : (c - n == r ? 1.0 : 0.0);
	for (int col = 0; col < n; col++) {
		int piv = col;
		for (int r = col + 1; r < n; r++)
			if (fabs(aug[r][col]) > fabs(aug[piv][col])) piv = r;
		if (piv != col)
			for (int c = 0; c < 2 * n; c++) {
				double t = aug[col][c]; aug[col][c] = aug[piv][c]; aug[piv][c] = t;
			}
		double inv = 1.0 / aug[col][col];
		for (int c = 0; c < 2 * n; c++) aug[col][c] *= inv;
		for (int r = 0; r < n; r++) {
			if (r == col) continue;
			double f = aug[r][col];
			if (f != 0.0)
				for (int c = 0; c < 2 * n; c++) aug[r][c] -= f * aug[col][c];
		}
	}
	for (int r = 0; r < n; r++)
		for (int c = 0; c < n; c++) A[r * n + c] = aug[r][n + c];
}

/* diff_tensor.c:1091-1162: inverse of the two-bead free-space RPY mobility,
 * returned in the same 18-component layout as JO_2B_R_matrix. */
static void orc_rpy_2b_resistance(double ai, double aj, double rx, double ry, double rz, double out[18])
{
	double Mij[6], A[36];
	static const int ra[6] = {0, 1, 2, 0, 0, 1};
	static const int cb[6] = {0, 1, 2, 1, 2, 2};
	orc_rpy_pair(ai, aj, rx, ry, rz, Mij);
	memset(A, 0, sizeof(A));
	for (int c = 0; c < 3; c++) {
		A[c * 6 + c] = 1.0 / (6 * ORC_PI * ai);
		A[(c + 3) * 6 + c + 3] = 1.0 / (6 * ORC_PI * aj);
	}
	for (int t = 0; t < 6; t++) {
		int r = ra[t], c = cb[t];
		A[r * 6 + c + 3] = A[c * 6 + r + 3] = Mij[t];
		A[(r + 3) * 6 + c] = A[(c + 3) * 6 + r] = Mij[t];
	}
	orc_invert_small(A, 6);
	for (int t = 0; t < 6; t++) {
		int r = ra[t], c = cb[t];
		out[t] = A[r * 6 + c];
		out[6 + t] = A[(r + 3) * 6 + c + 3];
		out[12 + t] = A[r * 6 + c + 3];
	}
}

/* diff_tensor.c:1166-1186: projection onto the relative-motion subspace. */
static void orc_cichocki(const double in[18], double out[18])
{
	for (int t = 0; t < 6; t++) {
		double self = (in[t] + in[6 + t] - 2 * in[12 + t]) / 4;
		out[t] = self;
		out[6 + t] = self;
		out[12 + t] = (2 * in[12 + t] - in[t] - in[6 + t]) / 4;
	}
}

/* diff_tensor.c:346-479: accumulates (+=) into a caller-zeroed 3N x 3N matrix. */
void JO_R_lubrication_correction_matrix(double *as, double *pointers, int number_of_beads,
                                        double cutoff_distance, int cichocki_correction,
                                        double *correction_matrix)
{
	int N = number_of_beads, n3 = 3 * N;
	for (int j = 0; j < N; j++) {
		for (int i = j + 1; i < N; i++) {
			const double *p = orc_pair_vec(pointers, i, j, N);
			double d = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
			if (!((d - as[j] - as[i]) / (as[j] + as[i]) <= cutoff_distance)) continue;
			double nf[18], ff[18], res[18];
			JO_2B_R_matrix(as[j], as[i], p[0], p[1], p[2], nf);
			orc_rpy_2b_resistance(as[j], as[i], p[0], p[1], p[2], ff);
			if (cichocki_correction) {
				double t[18];
				memcpy(t, nf, sizeof(t));
				orc_cichocki(t, nf);
				memcpy(t, ff, sizeof(t));
				orc_cichocki(t, ff);
			}
			for (int k = 0; k < 18; k++) res[k] = nf[k] - ff[k];
			orc_put_block(correction_matrix, n3, 3 * j, 3 * j, res, 1);
			orc_put_block(correction_matrix, n3, 3 * i, 3 * i, res + 6, 1);
			orc_put_block(correction_matrix, n3, 3 * i, 3 * j, res + 12, 1);
		}
	}
}
