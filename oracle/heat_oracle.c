/* ORACLE -- test infrastructure only (the checker and the timed CPU baseline; never part of
 * the product). C restatement of the heat-diffusion-2d update of
 * examples/heat-diffusion-2d/src/main.cc:408-421 (update_cpu) with DX = DY = 1 and
 * c = ALPHA*DT/(DX*DY), evaluated as ((S[i+1] - 2S) + S[i-1]) + ((S[j+1] - 2S) + S[j-1]) and
 * D = S + c*(that), compiled with -ffp-contract=off so no multiply-add is fused. Column-major
 * grids, cell (i, j) at G[j*ld + i]; only interior cells are written. Columns are split over
 * `nthreads` POSIX threads (the reference's host driver spreads tile tasks over its team). */
#include <pthread.h>
#include <stdint.h>

static inline double upd(double s, double up, double dn, double w, double e, double c)
{
    const double a = (dn - 2.0 * s) + up;
    const double b = (e - 2.0 * s) + w;
    return s + c * (a + b);
}

typedef struct { int kind; const void * src; void * dst; int64_t nx, ny, ld, j0, j1; double c, a, b; } job_t;

static void * run_job(void * p)
{
    const job_t * J = (const job_t *) p;
    if (J->kind == 0) {
        const double * src = (const double *) J->src; double * dst = (double *) J->dst;
        for (int64_t j = J->j0; j < J->j1; ++j) {
            const double * w = src + (j - 1) * J->ld, * s = src + j * J->ld, * e = src + (j + 1) * J->ld;
            double * d = dst + j * J->ld;
            for (int64_t i = 1; i < J->nx - 1; ++i) d[i] = upd(s[i], s[i - 1], s[i + 1], w[i], e[i], J->c);
        }
    } else if (J->kind == 1) {
        const float * src = (const float *) J->src; float * dst = (float *) J->dst;
        for (int64_t j = J->j0; j < J->j1; ++j) {
            const float * w = src + (j - 1) * J->ld, * s = src + j * J->ld, * e = src + (j + 1) * J->ld;
            float * d = dst + j * J->ld;
            for (int64_t i = 1; i < J->nx - 1; ++i) d[i] = (float) upd(s[i], s[i - 1], s[i + 1], w[i], e[i], J->c);
        }
    } else {
        const double * x = (const double *) J->src; double * y = (double *) J->dst;
        for (int64_t i = J->j0; i < J->j1; ++i) y[i] = (J->a * x[i]) + (J->b * y[i]);
    }
    return 0;
}

static void parallel(job_t base, int64_t lo, int64_t hi, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256]; job_t jobs[256];
    const int64_t n = hi - lo;
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = base;
        jobs[t].j0 = lo + n * t / nthreads; jobs[t].j1 = lo + n * (t + 1) / nthreads;
        if (t) pthread_create(&th[t], 0, run_job, &jobs[t]);
    }
    run_job(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(th[t], 0);
}

void xk_oracle_heat_step_f64(const double * src, double * dst, int64_t nx, int64_t ny, int64_t ld,
                             double c, int nthreads)
{
    job_t J = {0, src, dst, nx, ny, ld, 0, 0, c, 0, 0};
    if (nx >= 3 && ny >= 3) parallel(J, 1, ny - 1, nthreads);
}

void xk_oracle_heat_step_f32(const float * src, float * dst, int64_t nx, int64_t ny, int64_t ld,
                             double c, int nthreads)
{
    job_t J = {1, src, dst, nx, ny, ld, 0, 0, c, 0, 0};
    if (nx >= 3 && ny >= 3) parallel(J, 1, ny - 1, nthreads);
}

void xk_oracle_axpby(int64_t n, double a, const double * x, double b, double * y, int nthreads)
{
    job_t J = {2, x, y, 0, 0, 0, 0, 0, 0, a, b};
    parallel(J, 0, n, nthreads);
}
