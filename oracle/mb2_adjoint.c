/*
 * FP64 CPU reference of the BD window and its adjoint.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA adjoint
 * (mars_md_b200/csrc/mb2_adjoint.cu) and of the finite differences. The
 * reference code base has no adjoint; the forward model restated here in
 * double is the reference's BD step with tabulated forces:
 *   - pair force: TabulatedPotential::compute (TabulatedPotential.h:19-52) on
 *     the minimum-image distance (PeriodicBox.h:134-208), cut off beyond the
 *     interaction cutoff and below 1e-6 (Pairwise.h:214-304), all non-excluded
 *     pairs;
 *   - bond force: TabulatedBondComputer (BondComputer.h:136-192);
 *   - angle force: TabulatedAngleComputer + AngleGeometry (BondComputer.h:204-269,
 *     BondGeometry.h:13-45), periodic table;
 *   - update: x <- wrap(x + (D dt / kT) F + sqrt(2 D dt) xi) (BD.h:80-85).
 * The adjoint of one step is lambda_k = lambda_{k+1} + J(x_k)^T (c * lambda_{k+1})
 * with c = D dt / kT. Every force here is minus the gradient of a potential
 * that is piecewise linear in the distance or angle, so J is symmetric (except
 * where the angle's sine is floored at 1e-3) and J^T mu is computed as the
 * directional derivative of the force along mu. Table gradients use
 * dF/dU[h] = +step_inv, dF/dU[h+1] = -step_inv for the pair's bin h.
 */
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdlib.h>
#include <string.h>

typedef struct {
	const double* v;
	int size;
	double start;
	double step_inv;
	int periodic;
} adj_table;

typedef struct {
	int n;
	double L[3];
	double c[3]; /* D dt / kT per axis */
	double s[3]; /* sqrt(2 D dt) per axis */
	adj_table pair;
	double cutoff;
	const int* excl_off; /* CSR over particles, or NULL */
	const int* excl_nb;
	int excl_n;
	const int* bonds; /* (i, j) */
	int nb;
	adj_table bond;
	const int* angles; /* (i, j, k, pad) */
	int na;
	adj_table angle;
	/* 0: table bins, cutoffs and angle clamps decided in double. 1: decided
	 * with the reference's float arithmetic on the float-rounded coordinates
	 * (PeriodicBox::wrap_diff, Vector3::length2, sqrtf, TabulatedPotential's
	 * w = (x - start) * step_inv, AngleGeometry's cosine and acosf), as the
	 * float forward decides them; everything else stays double. With float
	 * states this gives the derivative of the map a float forward computes. */
	int float_bins;
	/* 0: every step's pairs are all pairs within the cutoff. k > 0: as the
	 * window's pairlist, the candidate pairs of step j are those within
	 * list_radius at step k * floor(j / k), the segment's start (the list the
	 * device builds at each checkpoint), tested against the cutoff at step j. */
	int list_every;
	double list_radius;
} adj_sys;

/* Dual number: value and derivative along one direction. */
typedef struct {
	double v, d;
} dual;

static dual dmk(double v, double d) {
	dual r = {v, d};
	return r;
}
static dual dadd(dual a, dual b) { return dmk(a.v + b.v, a.d + b.d); }
static dual dsub(dual a, dual b) { return dmk(a.v - b.v, a.d - b.d); }
static dual dmul(dual a, dual b) { return dmk(a.v * b.v, a.d * b.v + a.v * b.d); }
static dual ddiv(dual a, dual b) { return dmk(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
static dual dsqrt(dual a) {
	const double r = sqrt(a.v);
	return dmk(r, r > 0.0 ? a.d / (2.0 * r) : 0.0);
}
static dual dscale(dual a, double k) { return dmk(a.v * k, a.d * k); }

static double min_image(double x, double l) {
	const double image = floor(x * (1.0 / l));
	x -= image * l;
	return x >= 0.5 * l ? x - l : x;
}

static int excluded(const adj_sys* s, int a, int b) {
	if (!s->excl_off || a >= s->excl_n) return 0;
	for (int e = s->excl_off[a]; e < s->excl_off[a + 1]; ++e)
		if (s->excl_nb[e] == b) return 1;
	return 0;
}

/* PeriodicBox::wrap_diff_scalar in float (PeriodicBox.h:453-461). */
static float wrapf(float x, float l) {
	const float inv = 1.0f / l;
	const float image = floorf(x * inv);
	x = x - image * l;
	return x >= 0.5f * l ? x - l : x;
}

/* Minimum-image vector x_j - x_i and its length in the reference's float
 * arithmetic. */
static float float_dist(const adj_sys* s, const double* x, int i, int j, float r[3]) {
	for (int a = 0; a < 3; ++a) r[a] = wrapf((float)x[3 * j + a] - (float)x[3 * i + a], (float)s->L[a]);
	return sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

/* The table bin h of abscissa x (w = (x - start) * step_inv, floor) in float
 * or double arithmetic. */
static int table_home(const adj_table* t, double x, int in_float) {
	if (in_float) {
		const float w = ((float)x - (float)t->start) * (float)t->step_inv;
		return (int)floorf(w);
	}
	return (int)floor((x - t->start) * t->step_inv);
}

/* Table force F(x) = -dU/dx of the bin's linear interpolant; *bin = home
 * (or -1 where the force is constant 0: past the end of a non-periodic table).
 * in_float: the bin is decided in float arithmetic. */
static double table_force_at(const adj_table* t, double x, int in_float, int* bin, int* bin1) {
	int home = table_home(t, x, in_float);
	if (t->periodic) {
		home %= t->size;
		if (home < 0) home += t->size;
	} else {
		if (home >= t->size - 1) {
			*bin = -1;
			*bin1 = -1;
			return 0.0;
		}
		if (home < 0) home = 0;
	}
	const int home1 = t->periodic ? (home + 1) % t->size : home + 1;
	*bin = home;
	*bin1 = home1;
	return -(t->v[home1] - t->v[home]) * t->step_inv;
}

static double table_force(const adj_table* t, double x, int* bin, int* bin1) {
	return table_force_at(t, x, 0, bin, bin1);
}

/* Central-pair term (pair or bond): force on j is F(r) u, on i -F(r) u, with
 * u = (x_j - x_i) / r. With mu: tangent of the forces along mu (t), and the
 * table gradient mu . dforce/dU (g). */
static void radial_term(const adj_sys* s, const adj_table* tab, double cutoff, int i, int j,
						const double* x, double* f, const double* mu, double* t, double* g) {
	double r[3];
	for (int a = 0; a < 3; ++a) r[a] = min_image(x[3 * j + a] - x[3 * i + a], s->L[a]);
	const double d = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
	int h, h1;
	double F;
	if (s->float_bins) {
		/* The forward's float decisions: the pair's (i < j) float distance, the
		 * cutoff test dist * dist > rc * rc and the bin (Pairwise.h:214-304,
		 * BondComputer.h:168-191). */
		float rf[3];
		const float df = float_dist(s, x, i, j, rf);
		const float cf = (float)cutoff;
		if (df < 1e-6f || (cutoff > 0.0 && df * df > cf * cf)) return;
		F = table_force_at(tab, (double)df, 1, &h, &h1);
	} else {
		if (d < 1e-6 || (cutoff > 0.0 && d > cutoff)) return;
		F = table_force(tab, d, &h, &h1);
	}
	const double u[3] = {r[0] / d, r[1] / d, r[2] / d};
	if (f)
		for (int a = 0; a < 3; ++a) {
			f[3 * j + a] += F * u[a];
			f[3 * i + a] -= F * u[a];
		}
	if (mu) {
		double dv[3], ud = 0.0;
		for (int a = 0; a < 3; ++a) {
			dv[a] = mu[3 * j + a] - mu[3 * i + a];
			ud += u[a] * dv[a];
		}
		for (int a = 0; a < 3; ++a) {
			const double ta = F / d * (dv[a] - u[a] * ud);
			t[3 * j + a] += ta;
			t[3 * i + a] -= ta;
		}
		if (g && h >= 0) {
			g[h] += tab->step_inv * ud;
			g[h1] -= tab->step_inv * ud;
		}
	}
}

/* Angle term with forward-mode tangents along mu (AngleGeometry formula). */
static void angle_term(const adj_sys* s, int i, int j, int k, const double* x, double* f,
					   const double* mu, double* t) {
	dual ab[3], bc[3], ac[3];
	for (int a = 0; a < 3; ++a) {
		const double m_i = mu ? mu[3 * i + a] : 0.0, m_j = mu ? mu[3 * j + a] : 0.0,
					 m_k = mu ? mu[3 * k + a] : 0.0;
		ab[a] = dmk(min_image(x[3 * j + a] - x[3 * i + a], s->L[a]), m_j - m_i);
		bc[a] = dmk(min_image(x[3 * k + a] - x[3 * j + a], s->L[a]), m_k - m_j);
		ac[a] = dmk(min_image(x[3 * k + a] - x[3 * i + a], s->L[a]), m_k - m_i);
	}
	const dual ab2 = dadd(dadd(dmul(ab[0], ab[0]), dmul(ab[1], ab[1])), dmul(ab[2], ab[2]));
	const dual bc2 = dadd(dadd(dmul(bc[0], bc[0]), dmul(bc[1], bc[1])), dmul(bc[2], bc[2]));
	const dual ac2 = dadd(dadd(dmul(ac[0], ac[0]), dmul(ac[1], ac[1])), dmul(ac[2], ac[2]));
	const dual lab = dsqrt(ab2), lbc = dsqrt(bc2);
	dual cs = ddiv(dscale(dsub(dadd(ab2, bc2), ac2), 0.5), dmul(lab, lbc));
	int h, h1;
	double F;
	dual sn;
	if (s->float_bins) {
		/* AngleGeometry (BondGeometry.h:19-44) in float: cosine by the law of
		 * cosines, clamps, acosf, the sine floor, the periodic table bin. */
		float rab[3], rbc[3], rac[3];
		const float lab_f = float_dist(s, x, i, j, rab), lbc_f = float_dist(s, x, j, k, rbc);
		float_dist(s, x, i, k, rac);
		const float ab2f = rab[0] * rab[0] + rab[1] * rab[1] + rab[2] * rab[2];
		const float bc2f = rbc[0] * rbc[0] + rbc[1] * rbc[1] + rbc[2] * rbc[2];
		const float ac2f = rac[0] * rac[0] + rac[1] * rac[1] + rac[2] * rac[2];
		float csf = (ab2f + bc2f - ac2f) * 0.5f / (lab_f * lbc_f);
		if (csf < -1.0f) {
			csf = -1.0f;
			cs = dmk(-1.0, 0.0);
		}
		if (csf > 1.0f) {
			csf = 1.0f;
			cs = dmk(1.0, 0.0);
		}
		sn = dsqrt(dsub(dmk(1.0, 0.0), dmul(cs, cs)));
		if (sqrtf(1.0f - csf * csf) <= 1e-3f) sn = dmk(1e-3, 0.0);
		F = table_force_at(&s->angle, (double)acosf(csf), 1, &h, &h1);
	} else {
		if (cs.v < -1.0) cs = dmk(-1.0, 0.0);
		if (cs.v > 1.0) cs = dmk(1.0, 0.0);
		const double angle = acos(cs.v);
		sn = dsqrt(dsub(dmk(1.0, 0.0), dmul(cs, cs)));
		if (sn.v <= 1e-3) sn = dmk(1e-3, 0.0);
		F = table_force(&s->angle, angle, &h, &h1);
	}
	const dual dudt = ddiv(dmk(-F, 0.0), sn);
	const dual inv_ab = ddiv(dmk(1.0, 0.0), lab), inv_bc = ddiv(dmk(1.0, 0.0), lbc);
	const dual s1 = dmul(dudt, inv_ab), c_ab = dmul(cs, inv_ab);
	const dual s3 = dscale(dmul(dudt, inv_bc), -1.0), c_bc = dmul(cs, inv_bc);
	for (int a = 0; a < 3; ++a) {
		const dual f1 = dmul(s1, dadd(dmul(ab[a], c_ab), dmul(bc[a], inv_bc)));
		const dual f3 = dmul(s3, dadd(dmul(bc[a], c_bc), dmul(ab[a], inv_ab)));
		if (f) {
			f[3 * i + a] += f1.v;
			f[3 * j + a] -= f1.v + f3.v;
			f[3 * k + a] += f3.v;
		}
		if (t) {
			t[3 * i + a] += f1.d;
			t[3 * j + a] -= f1.d + f3.d;
			t[3 * k + a] += f3.d;
		}
	}
}

/* Candidate pairs (i < j, not excluded) whose minimum-image distance may be
 * within rmax: a periodic cell list with cells at least rmax wide when every
 * axis holds three or more of them, else all pairs. Each caller applies its
 * own exact distance test, so the candidate set only has to contain every pair
 * within rmax. Threads take contiguous ranges of i and their lists are joined
 * in thread order, so the order is fixed for a given thread count. Returns the
 * count; *out (i, j) is malloc'd, the caller frees. */
static size_t near_pairs(const adj_sys* s, const double* x, double rmax, int** out) {
	const int n = s->n;
	int nc[3];
	int cells_ok = 1;
	for (int a = 0; a < 3; ++a) {
		nc[a] = (int)floor(s->L[a] / rmax);
		if (nc[a] < 3) cells_ok = 0;
	}
	if (!cells_ok) nc[0] = nc[1] = nc[2] = 1;
	const size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
	int* cell_of = (int*)malloc(sizeof(int) * (size_t)(n ? n : 1));
	int* start = (int*)calloc(ncell + 1, sizeof(int));
	int* members = (int*)malloc(sizeof(int) * (size_t)(n ? n : 1));
	for (int i = 0; i < n; ++i) {
		int c[3];
		for (int a = 0; a < 3; ++a) {
			double u = x[3 * i + a] / s->L[a];
			u -= floor(u);
			c[a] = (int)(u * nc[a]);
			if (c[a] >= nc[a]) c[a] = nc[a] - 1;
			if (c[a] < 0) c[a] = 0;
		}
		cell_of[i] = (c[0] * nc[1] + c[1]) * nc[2] + c[2];
		++start[cell_of[i] + 1];
	}
	for (size_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
	int* fill = (int*)malloc(sizeof(int) * ncell);
	for (size_t c = 0; c < ncell; ++c) fill[c] = start[c];
	for (int i = 0; i < n; ++i) members[fill[cell_of[i]]++] = i;
	free(fill);
	int nthreads = 1;
#ifdef _OPENMP
	nthreads = omp_get_max_threads();
#endif
	int** tp = (int**)calloc((size_t)nthreads, sizeof(int*));
	size_t* tc = (size_t*)calloc((size_t)nthreads, sizeof(size_t));
#pragma omp parallel num_threads(nthreads)
	{
		int tid = 0;
#ifdef _OPENMP
		tid = omp_get_thread_num();
#endif
		size_t cap = 1024, cnt = 0;
		int* p = (int*)malloc(sizeof(int) * 2 * cap);
#pragma omp for schedule(static)
		for (int i = 0; i < n; ++i) {
			const int ci = cell_of[i];
			const int cx = ci / (nc[1] * nc[2]), cy = (ci / nc[2]) % nc[1], cz = ci % nc[2];
			const int span = cells_ok ? 1 : 0;
			for (int dx = -span; dx <= span; ++dx)
				for (int dy = -span; dy <= span; ++dy)
					for (int dz = -span; dz <= span; ++dz) {
						const int ox = (cx + dx + nc[0]) % nc[0], oy = (cy + dy + nc[1]) % nc[1],
								  oz = (cz + dz + nc[2]) % nc[2];
						const int c = (ox * nc[1] + oy) * nc[2] + oz;
						for (int q = start[c]; q < start[c + 1]; ++q) {
							const int j = members[q];
							if (j <= i || excluded(s, i, j)) continue;
							if (cnt == cap) {
								cap *= 2;
								p = (int*)realloc(p, sizeof(int) * 2 * cap);
							}
							p[2 * cnt] = i;
							p[2 * cnt + 1] = j;
							++cnt;
						}
					}
		}
		tp[tid] = p;
		tc[tid] = cnt;
	}
	size_t total = 0;
	for (int t = 0; t < nthreads; ++t) total += tc[t];
	int* all = (int*)malloc(sizeof(int) * 2 * (total ? total : 1));
	size_t at = 0;
	for (int t = 0; t < nthreads; ++t) {
		if (tc[t]) memcpy(all + 2 * at, tp[t], sizeof(int) * 2 * tc[t]);
		at += tc[t];
		free(tp[t]);
	}
	free(tp);
	free(tc);
	free(cell_of);
	free(start);
	free(members);
	*out = all;
	return total;
}

/* Adds thread-private accumulators into the shared ones in thread order. */
static void add_into(double* dst, const double* src, size_t len) {
	if (!dst) return;
	for (size_t q = 0; q < len; ++q) dst[q] += src[q];
}

/* Total force (f) and, when mu is given, its tangent along mu (t) and the
 * table gradients (gpair, gbond: mu . dforce/dU, accumulated). */
/* Pairs within list_radius of each other at x (the float test of the
 * device's list build when float_bins, else double): a segment's pairlist. */
static size_t list_pairs(const adj_sys* s, const double* x, int** out) {
	int* cand = NULL;
	const size_t nc = near_pairs(s, x, s->list_radius, &cand);
	size_t k = 0;
	const float rl = (float)s->list_radius;
	for (size_t q = 0; q < nc; ++q) {
		const int i = cand[2 * q], j = cand[2 * q + 1];
		int keep;
		if (s->float_bins) {
			float r[3];
			for (int a = 0; a < 3; ++a)
				r[a] = wrapf((float)x[3 * j + a] - (float)x[3 * i + a], (float)s->L[a]);
			keep = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] <= rl * rl;
		} else {
			double d2 = 0.0;
			for (int a = 0; a < 3; ++a) {
				const double d = min_image(x[3 * j + a] - x[3 * i + a], s->L[a]);
				d2 += d * d;
			}
			keep = d2 <= s->list_radius * s->list_radius;
		}
		if (keep) {
			cand[2 * k] = i;
			cand[2 * k + 1] = j;
			++k;
		}
	}
	*out = cand;
	return k;
}

/* The candidate pairs of step k of a trajectory under s->list_every, kept in
 * *cache (built for segment *cache_k0). */
static const int* step_pairs(const adj_sys* s, const double* traj, int k, int* cache_k0,
							 int** cache, size_t* np) {
	const size_t m = 3 * (size_t)s->n;
	const int k0 = (k / s->list_every) * s->list_every;
	if (*cache == NULL || *cache_k0 != k0) {
		free(*cache);
		*np = list_pairs(s, traj + (size_t)k0 * m, cache);
		*cache_k0 = k0;
	}
	return *cache;
}

static void forces_on(const adj_sys* s, const double* x, double* f, const double* mu, double* t,
					  double* gpair, double* gbond, const int* list, size_t nlist);

static void forces(const adj_sys* s, const double* x, double* f, const double* mu, double* t,
				   double* gpair, double* gbond) {
	forces_on(s, x, f, mu, t, gpair, gbond, NULL, 0);
}

/* forces() over the candidate pairs `list` (all pairs within the cutoff when
 * NULL); each candidate is tested against the cutoff at x. */
static void forces_on(const adj_sys* s, const double* x, double* f, const double* mu, double* t,
					  double* gpair, double* gbond, const int* list, size_t nlist) {
	int* pr = NULL;
	size_t np;
	if (list) {
		np = nlist;
	} else {
		np = near_pairs(s, x, s->cutoff, &pr);
		list = pr;
	}
	const size_t m = 3 * (size_t)s->n, gs = (size_t)s->pair.size;
	int nthreads = 1;
#ifdef _OPENMP
	nthreads = omp_get_max_threads();
#endif
	double** acc = (double**)calloc((size_t)nthreads, sizeof(double*));
#pragma omp parallel num_threads(nthreads)
	{
		int tid = 0;
#ifdef _OPENMP
		tid = omp_get_thread_num();
#endif
		double* buf = (double*)calloc(2 * m + gs + 1, sizeof(double));
		double* fl = f ? buf : NULL;
		double* tl = t ? buf + m : NULL;
		double* gl = gpair ? buf + 2 * m : NULL;
#pragma omp for schedule(static)
		for (size_t q = 0; q < np; ++q)
			radial_term(s, &s->pair, s->cutoff, list[2 * q], list[2 * q + 1], x, fl, mu, tl, gl);
		acc[tid] = buf;
	}
	for (int th = 0; th < nthreads; ++th) {
		add_into(f, acc[th], m);
		add_into(t, acc[th] + m, m);
		add_into(gpair, acc[th] + 2 * m, gs);
		free(acc[th]);
	}
	free(acc);
	free(pr);
	for (int b = 0; b < s->nb; ++b)
		radial_term(s, &s->bond, 0.0, s->bonds[2 * b], s->bonds[2 * b + 1], x, f, mu, t, gbond);
	for (int a = 0; a < s->na; ++a)
		angle_term(s, s->angles[4 * a], s->angles[4 * a + 1], s->angles[4 * a + 2], x, f, mu, t);
}

void adj_forces64(const adj_sys* s, const double* x, double* f) {
	memset(f, 0, sizeof(double) * 3 * (size_t)s->n);
	forces(s, x, f, NULL, NULL, NULL, NULL);
}

/* traj: (steps + 1) * n * 3, traj[0] = x0; noise: steps * n * 3 normals. */
void adj_forward64(const adj_sys* s, const double* x0, const double* noise, int steps,
				   double* traj) {
	const size_t m = 3 * (size_t)s->n;
	double* f = (double*)malloc(sizeof(double) * m);
	int* cache = NULL;
	int cache_k0 = -1;
	size_t np = 0;
	memcpy(traj, x0, sizeof(double) * m);
	for (int k = 0; k < steps; ++k) {
		const double* x = traj + (size_t)k * m;
		double* y = traj + (size_t)(k + 1) * m;
		memset(f, 0, sizeof(double) * m);
		if (s->list_every > 0) {
			const int* list = step_pairs(s, traj, k, &cache_k0, &cache, &np);
			forces_on(s, x, f, NULL, NULL, NULL, NULL, list, np);
		} else {
			forces(s, x, f, NULL, NULL, NULL, NULL);
		}
		for (size_t q = 0; q < m; ++q) {
			const int a = (int)(q % 3);
			double v = x[q] + s->c[a] * f[q] + s->s[a] * noise[(size_t)k * m + q];
			v -= s->L[a] * floor(v / s->L[a]);
			y[q] = v;
		}
	}
	free(cache);
	free(f);
}

/* lam: in lambda_N, out lambda_0; gpair / gbond accumulated. */
void adj_backward64(const adj_sys* s, const double* traj, int steps, double* lam, double* gpair,
					double* gbond) {
	const size_t m = 3 * (size_t)s->n;
	double* mu = (double*)calloc(m ? m : 1, sizeof(double));
	double* t = (double*)malloc(sizeof(double) * m);
	int* cache = NULL;
	int cache_k0 = -1;
	size_t np = 0;
	for (int k = steps - 1; k >= 0; --k) {
		for (size_t q = 0; q < m; ++q) mu[q] = s->c[q % 3] * lam[q];
		memset(t, 0, sizeof(double) * m);
		if (s->list_every > 0) {
			const int* list = step_pairs(s, traj, k, &cache_k0, &cache, &np);
			forces_on(s, traj + (size_t)k * m, NULL, mu, t, gpair, gbond, list, np);
		} else {
			forces(s, traj + (size_t)k * m, NULL, mu, t, gpair, gbond);
		}
		for (size_t q = 0; q < m; ++q) lam[q] += t[q];
	}
	free(cache);
	free(mu);
	free(t);
}

/* Gaussian-smoothed pair-distance histogram over non-excluded pairs with
 * r < rmax: hist[b] += exp(-(r - r_b)^2 / (2 sigma^2)) for |r - r_b| <= 5 sigma,
 * r_b = (b + 1/2) dr. */
void adj_rdf64(const adj_sys* s, const double* x, int nbins, double dr, double rmax, double sigma,
			   double* hist) {
	memset(hist, 0, sizeof(double) * (size_t)nbins);
	int* pr = NULL;
	const size_t np = near_pairs(s, x, rmax, &pr);
	for (size_t q = 0; q < np; ++q) {
		const int i = pr[2 * q], j = pr[2 * q + 1];
		{
			double r2 = 0.0;
			for (int a = 0; a < 3; ++a) {
				const double d = min_image(x[3 * j + a] - x[3 * i + a], s->L[a]);
				r2 += d * d;
			}
			const double r = sqrt(r2);
			if (!(r < rmax)) continue;
			for (int b = 0; b < nbins; ++b) {
				const double z = r - (b + 0.5) * dr;
				if (fabs(z) <= 5.0 * sigma) hist[b] += exp(-z * z / (2.0 * sigma * sigma));
			}
		}
	}
	free(pr);
}

/* grad (n * 3, accumulated) of sum_b dLdh[b] hist[b] with respect to x. */
void adj_rdf_grad64(const adj_sys* s, const double* x, int nbins, double dr, double rmax,
					double sigma, const double* dLdh, double* grad) {
	int* pr = NULL;
	const size_t np = near_pairs(s, x, rmax, &pr);
	for (size_t q = 0; q < np; ++q) {
		const int i = pr[2 * q], j = pr[2 * q + 1];
		{
			double r[3], r2 = 0.0;
			for (int a = 0; a < 3; ++a) {
				r[a] = min_image(x[3 * j + a] - x[3 * i + a], s->L[a]);
				r2 += r[a] * r[a];
			}
			const double d = sqrt(r2);
			if (!(d < rmax) || d < 1e-12) continue;
			double dLdr = 0.0;
			for (int b = 0; b < nbins; ++b) {
				const double z = d - (b + 0.5) * dr;
				if (fabs(z) <= 5.0 * sigma)
					dLdr += dLdh[b] * exp(-z * z / (2.0 * sigma * sigma)) * (-z / (sigma * sigma));
			}
			for (int a = 0; a < 3; ++a) {
				grad[3 * j + a] += dLdr * r[a] / d;
				grad[3 * i + a] -= dLdr * r[a] / d;
			}
		}
	}
	free(pr);
}
