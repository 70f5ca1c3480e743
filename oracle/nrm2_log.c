/* Residual-history tap for the reference oracle (test infrastructure only).
 *
 * The reference solvers report nothing but their final iteration index.
 * Every convergence test they make, however, is a cblas_dnrm2 call
 * (e.g. src/bicgstabl.c:122 `error = cblas_dnrm2(n, r[0], 1) / fnb`), and
 * the first dnrm2 each solver makes is ||b|| (src/cg.c:30, src/bicgstabl.c:51,
 * src/blcg.c:60, ...).  Linking the reference sources with
 * -Wl,--wrap=cblas_dnrm2 routes those calls through this file, which records
 * each returned norm into a caller-supplied buffer, so the history of
 * recursive residual norms can be compared without editing the reference. */
double __real_cblas_dnrm2(const int n, const double *x, const int incx);

static double *g_buf = 0;
static int g_cap = 0;
static int g_len = 0;

double __wrap_cblas_dnrm2(const int n, const double *x, const int incx)
{
    double v = __real_cblas_dnrm2(n, x, incx);
    if (g_buf && g_len < g_cap)
        g_buf[g_len] = v;
    if (g_buf)
        g_len++;
    return v;
}

/* The complex solvers' norms (src/bicg.c:159, src/bicgstabl.c:259, ...)
 * go through cblas_dznrm2; they are recorded into the same buffer. */
double __real_cblas_dznrm2(const int n, const void *x, const int incx);

double __wrap_cblas_dznrm2(const int n, const void *x, const int incx)
{
    double v = __real_cblas_dznrm2(n, x, incx);
    if (g_buf && g_len < g_cap)
        g_buf[g_len] = v;
    if (g_buf)
        g_len++;
    return v;
}

/* Zero-filled allocation for the reference's workspaces.
 *
 * dblcg reads its s-by-s beta block before writing the off-diagonal entries
 * (src/blcg.c:32-34 malloc, :61-63 sets only the diagonal, :68 reads it), so
 * its result depends on what malloc happens to return: in a fresh process
 * the pages are zero and beta = I; inside a long-running process it is
 * garbage and the solve returns NaN.  Linking with -Wl,--wrap=malloc routes
 * the reference's malloc calls here, pinning the intended beta = I without
 * editing the reference. */
void *calloc(unsigned long nmemb, unsigned long size);
void *__wrap_malloc(unsigned long size)
{
    return calloc(1, size ? size : 1);
}

/* Start recording into buf[0..cap). */
void oracle_nrm2_log_begin(double *buf, int cap)
{
    g_buf = buf;
    g_cap = cap;
    g_len = 0;
}

/* Stop recording; returns how many norms were produced (may exceed cap). */
int oracle_nrm2_log_end(void)
{
    int n = g_len;
    g_buf = 0;
    g_cap = 0;
    g_len = 0;
    return n;
}
