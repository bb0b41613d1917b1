/*
 * cpu_rk4.c -- FP64 CPU restatement of SLOTH's ray trace with a fixed-step
 * fourth-order Runge-Kutta(-Nystrom) integrator, the method of the CUDA tracers.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA tracers and the timed
 * CPU baseline. Nothing in the product links or calls it.
 *
 * Follows (paths relative to the SLOTH repo):
 *   dsdt                src/core/propagator.py:168-243  dr/dt = v, dv/dt = grad G(r),
 *                                                       dtau/dt = kappa(r)
 *   interpolator        src/core/interpolator.py:79-104 trilinear, fill 0 outside
 *                       (the uniform-grid form of searchsorted-1 clamped to [0, n-2])
 *   phase integrand     src/legacy/full_solver.py:271-274, :289, :341-347  omega*(n - 1),
 *                       n - 1 interpolated from its grid values (fill 0 outside, i.e. n = 1)
 *   keep_current_plane  src/shared/propagation.py:4-90
 * The grid fields (ne and the three gradient grids of G, kappa, n - 1) come
 * from the numpy restatement of precompute_gradients / kappa_inv_brems /
 * n_refrac, in SI units.
 * Same semantics as trace_rays() in ref_restated.py, written independently
 * in C for speed (pthreads over rays, 64-ray chunks from an atomic counter).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORACLE_C 299792458.0
#define FACE_MARGIN 0.02   /* cells: steps ending this close to a face sample the inside limit */

typedef struct {
    int32_t n[3];
    int32_t pad;
    double origin[3];
    double spacing[3];
    const double* fields;   /* (nx,ny,nz,4): ne, dG/dx, dG/dy, dG/dz */
    const double* kappa;    /* (nx,ny,nz) or NULL */
    double omega;
    double dt;              /* seconds */
    int32_t first_save, save_every, n_saves;
    int32_t axis, project;
    int32_t inv_brems, early_exit;
    int32_t threads;        /* <= 0: all online cores */
    double plane;
    int32_t integrator;     /* 0: Runge-Kutta-Nystrom (3 samples), 1: classical RK4 (4 samples) */
    int32_t pad2;
    const double* nm1;      /* (nx,ny,nz) n - 1 of the plasma refractive index */
} OracleParams;

typedef struct {
    double f[4];
    double k, m;            /* kappa, n - 1 */
} Samp;

/* clip != 0 clamps the point into the grid in cell units first: a clamp in
 * metres can map back to a cell coordinate just above n - 1 by rounding, and
 * then sample the fill value instead of the field's limit from inside. */
static void sample(const OracleParams* p, const double r[3], int clip, Samp* s) {
    double u[3], t[3];
    int i[3];
    for (int a = 0; a < 3; ++a) {
        u[a] = (r[a] - p->origin[a]) / p->spacing[a];
        if (clip) u[a] = u[a] < 0.0 ? 0.0 : (u[a] > (double)(p->n[a] - 1) ? (double)(p->n[a] - 1) : u[a]);
        if (!(u[a] >= 0.0 && u[a] <= (double)(p->n[a] - 1))) {
            memset(s, 0, sizeof(*s));
            return;
        }
        int k = (int)floor(u[a]);
        if (k > p->n[a] - 2) k = p->n[a] - 2;
        i[a] = k;
        t[a] = u[a] - (double)k;
    }
    const size_t sy = (size_t)p->n[2], sx = (size_t)p->n[1] * (size_t)p->n[2];
    memset(s, 0, sizeof(*s));
    /* corner order of itertools.product: z fastest */
    for (int e0 = 0; e0 < 2; ++e0)
        for (int e1 = 0; e1 < 2; ++e1)
            for (int e2 = 0; e2 < 2; ++e2) {
                double w = 1.0;
                w *= e0 ? t[0] : 1.0 - t[0];
                w *= e1 ? t[1] : 1.0 - t[1];
                w *= e2 ? t[2] : 1.0 - t[2];
                const size_t v = (size_t)(i[0] + e0) * sx + (size_t)(i[1] + e1) * sy + (size_t)(i[2] + e2);
                const double* f = p->fields + 4 * v;
                s->f[0] += f[0] * w;
                s->f[1] += f[1] * w;
                s->f[2] += f[2] * w;
                s->f[3] += f[3] * w;
                if (p->kappa) s->k += p->kappa[v] * w;
                s->m += p->nm1[v] * w;
            }
}

static void rhs(const OracleParams* p, const double r[3], int clip, double a[3], double* g, double* k) {
    Samp s;
    sample(p, r, clip, &s);   /* a step cut at a face samples the field's limit from inside */
    a[0] = s.f[1];
    a[1] = s.f[2];
    a[2] = s.f[3];
    *g = p->omega * s.m;   /* omega * (interpolated n - 1), 0 outside */
    *k = p->inv_brems ? s.k : 0.0;
}

static int gone(const OracleParams* p, const double r[3], const double v[3]) {
    for (int a = 0; a < 3; ++a) {
        const double lo = p->origin[a], hi = p->origin[a] + p->spacing[a] * (double)(p->n[a] - 1);
        if ((r[a] < lo && v[a] <= 0.0) || (r[a] > hi && v[a] >= 0.0)) return 1;
    }
    return 0;
}

static void jones_of(const OracleParams* p, const double x[3], const double v[3], double out[4]) {
    const int ax = p->axis, t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
    double p1 = x[t1], p2 = x[t2];
    if (p->project) {
        const double tbp = (x[ax] - p->plane) / v[ax];
        p1 = x[t1] - v[t1] * tbp;
        p2 = x[t2] - v[t2] * tbp;
    }
    out[0] = p1;
    out[1] = atan(v[t1] / v[ax]);
    out[2] = p2;
    out[3] = atan(v[t2] / v[ax]);
}

/* Outputs ([S][rows][N] row-major, any may be NULL):
 * state [S][6][N], jones [S][4][N], phase [S][N], tau [S][N], steps [N], status [N]. */
typedef struct {
    const OracleParams* p;
    const double* rays;
    int64_t n;
    double *state, *jones, *phase, *tau;
    int32_t* steps;
    uint8_t* status;
    int64_t next;       /* atomic work counter */
    long long total;    /* atomic ray-step total */
} Job;

static int inside(const OracleParams* p, const double r[3]) {
    for (int a = 0; a < 3; ++a) {
        const double lo = p->origin[a], hi = p->origin[a] + p->spacing[a] * (double)(p->n[a] - 1);
        if (!(r[a] >= lo && r[a] <= hi)) return 0;
    }
    return 1;
}

/* One step of length h (seconds) of r'' = grad G(r) with phase' = g(r) and
 * tau' = kappa(r): Nystrom's fourth-order Runge-Kutta-Nystrom method (three
 * samples), with Simpson's weights for the two integrals:
 *   r2 = r + h/2 v + h^2/8 a1,  r3 = r + h v + h^2/2 a2,
 *   r' = r + h v + h^2/6 (a1 + 2 a2),  v' = v + h/6 (a1 + 4 a2 + a3). */
static void step_rkn(const OracleParams* p, double h, int clip, double r[3], double v[3], double* ph, double* ta) {
    double a1[3], a2[3], a3[3], r2[3], r3[3];
    double g1, g2, g3, k1, k2, k3;
    rhs(p, r, clip, a1, &g1, &k1);
    for (int a = 0; a < 3; ++a) r2[a] = r[a] + 0.5 * h * v[a] + (h * h / 8.0) * a1[a];
    rhs(p, r2, clip, a2, &g2, &k2);
    for (int a = 0; a < 3; ++a) r3[a] = r[a] + h * v[a] + (h * h / 2.0) * a2[a];
    rhs(p, r3, clip, a3, &g3, &k3);
    for (int a = 0; a < 3; ++a) {
        r[a] = r[a] + h * v[a] + (h * h / 6.0) * (a1[a] + 2.0 * a2[a]);
        v[a] = v[a] + h / 6.0 * (a1[a] + 4.0 * a2[a] + a3[a]);
    }
    *ph += h / 6.0 * (g1 + 4.0 * g2 + g3);
    *ta += h / 6.0 * (k1 + 4.0 * k2 + k3);
}

/* One classical RK4 step of length h of the first-order system (r, v)' =
 * (v, grad G(r)) with the phase and the depth on RK4's weights:
 *   r2 = r + h/2 v, v2 = v + h/2 a1;  r3 = r + h/2 v2, v3 = v + h/2 a2;
 *   r4 = r + h v3, v4 = v + h a3;  r' = r + h/6 (v + 2 v2 + 2 v3 + v4),
 *   v' = v + h/6 (a1 + 2 a2 + 2 a3 + a4). */
static void step_rk4(const OracleParams* p, double h, int clip, double r[3], double v[3], double* ph, double* ta) {
    double a1[3], a2[3], a3[3], a4[3], r2[3], v2[3], r3[3], v3[3], r4[3], v4[3];
    double g1, g2, g3, g4, k1, k2, k3, k4;
    rhs(p, r, clip, a1, &g1, &k1);
    for (int a = 0; a < 3; ++a) {
        r2[a] = r[a] + 0.5 * h * v[a];
        v2[a] = v[a] + 0.5 * h * a1[a];
    }
    rhs(p, r2, clip, a2, &g2, &k2);
    for (int a = 0; a < 3; ++a) {
        r3[a] = r[a] + 0.5 * h * v2[a];
        v3[a] = v[a] + 0.5 * h * a2[a];
    }
    rhs(p, r3, clip, a3, &g3, &k3);
    for (int a = 0; a < 3; ++a) {
        r4[a] = r[a] + h * v3[a];
        v4[a] = v[a] + h * a3[a];
    }
    rhs(p, r4, clip, a4, &g4, &k4);
    for (int a = 0; a < 3; ++a) {
        r[a] += h / 6.0 * (v[a] + 2.0 * v2[a] + 2.0 * v3[a] + v4[a]);
        v[a] += h / 6.0 * (a1[a] + 2.0 * a2[a] + 2.0 * a3[a] + a4[a]);
    }
    *ph += h / 6.0 * (g1 + 2.0 * g2 + 2.0 * g3 + g4);
    *ta += h / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
}

/* A ray inside the grid whose straight-line prediction leaves it within the
 * step takes a step shortened to the face (the RHS is discontinuous there)
 * and is then frozen at time step + phi; a ray outside on an axis and moving
 * away on it is frozen at once (early_exit) or stepped with the zero RHS. */
static long long trace_one(const OracleParams* p, const double* rays, int64_t n, int64_t id, double* state,
                           double* jones, double* phase, double* tau, int32_t* steps, uint8_t* status) {
    const int S = p->n_saves;
    const int every = S > 1 ? p->save_every : 0;
    const long long last = (long long)p->first_save + (long long)(S - 1) * every;
    const double dt = p->dt;
    double r[3], v[3];
    for (int a = 0; a < 3; ++a) {
        r[a] = rays[a * n + id];
        v[a] = rays[(3 + a) * n + id];
    }
    double ph = 0.0, ta = 0.0, frozen_t = -1.0;
    long long step = 0, nst = 0, next_save = p->first_save;
    int j = 0;
    for (;;) {
        while (j < S && next_save == step) {
            const double drift = frozen_t >= 0.0 ? ((double)step - frozen_t) * dt : 0.0;
            double xs[3];
            for (int a = 0; a < 3; ++a) xs[a] = r[a] + v[a] * drift;
            if (state)
                for (int a = 0; a < 3; ++a) {
                    state[((size_t)j * 6 + a) * n + id] = xs[a];
                    state[((size_t)j * 6 + 3 + a) * n + id] = v[a];
                }
            if (jones) {
                double o[4];
                jones_of(p, xs, v, o);
                for (int k = 0; k < 4; ++k) jones[((size_t)j * 4 + k) * n + id] = o[k];
            }
            if (phase) phase[(size_t)j * n + id] = ph;
            if (tau) tau[(size_t)j * n + id] = ta;
            ++j;
            next_save += every;
        }
        if (j >= S || step > last) break;
        if (frozen_t < 0.0 && p->early_exit && gone(p, r, v)) frozen_t = (double)step;
        if (frozen_t < 0.0) {
            double phi = 1.0;
            int near = 0;
            if (inside(p, r)) {
                for (int a = 0; a < 3; ++a) {
                    const double lo = p->origin[a], hi = p->origin[a] + p->spacing[a] * (double)(p->n[a] - 1);
                    const double pn = r[a] + v[a] * dt;
                    const double marg = FACE_MARGIN * p->spacing[a];
                    if (pn > hi - marg || pn < lo + marg) near = 1;
                    if (pn > hi) {
                        const double t = (hi - r[a]) / (v[a] * dt);
                        if (t < phi) phi = t;
                    }
                    if (pn < lo) {
                        const double t = (lo - r[a]) / (v[a] * dt);
                        if (t < phi) phi = t;
                    }
                }
            }
            const int split = phi < 1.0;
            if (phi < 0.0) phi = 0.0;
            if (p->integrator == 1)
                step_rk4(p, dt * phi, split || near, r, v, &ph, &ta);
            else
                step_rkn(p, dt * phi, split || near, r, v, &ph, &ta);
            ++nst;
            if (split) frozen_t = (double)step + phi;
        }
        ++step;
    }
    if (steps) steps[id] = (int32_t)nst;
    if (status) {
        int finite = isfinite(ph);
        for (int a = 0; a < 3; ++a) finite &= isfinite(r[a]) && isfinite(v[a]);
        status[id] = !finite ? 2 : ((frozen_t < 0.0 && inside(p, r)) ? 1 : 0);
    }
    return nst;
}

static void* worker(void* arg) {
    Job* jb = (Job*)arg;
    long long local = 0;
    for (;;) {
        const int64_t start = __atomic_fetch_add(&jb->next, 64, __ATOMIC_RELAXED);
        if (start >= jb->n) break;
        const int64_t end = start + 64 < jb->n ? start + 64 : jb->n;
        for (int64_t id = start; id < end; ++id)
            local += trace_one(jb->p, jb->rays, jb->n, id, jb->state, jb->jones, jb->phase, jb->tau,
                               jb->steps, jb->status);
    }
    __atomic_fetch_add(&jb->total, local, __ATOMIC_RELAXED);
    return NULL;
}

int oracle_threads(void) {
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

int oracle_trace(const OracleParams* p, const double* rays, int64_t n, double* state, double* jones,
                 double* phase, double* tau, int32_t* steps, uint8_t* status,
                 long long* total_steps) {
    if (!p || !rays || n < 0 || p->n_saves < 1) return -1;
    Job jb = {p, rays, n, state, jones, phase, tau, steps, status, 0, 0};
    int nt = p->threads > 0 ? p->threads : oracle_threads();
    if (nt > 1024) nt = 1024;
    if ((int64_t)nt > (n + 63) / 64) nt = (int)((n + 63) / 64);
    if (nt <= 1) {
        worker(&jb);
    } else {
        pthread_t th[1024];
        int started = 0;
        for (int t = 0; t < nt; ++t) {
            if (pthread_create(&th[t], NULL, worker, &jb) != 0) break;
            ++started;
        }
        if (started == 0) worker(&jb);
        for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
    }
    if (total_steps) *total_steps = jb.total;
    return 0;
}
