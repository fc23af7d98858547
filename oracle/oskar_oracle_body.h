/*
 * Precision-generic body of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 * Included twice by oskar_oracle.c with REAL/S/ORC_SIN/... defined for
 * double and for float. Each function states the reference code it restates.
 */

typedef struct { REAL re, im; } ORC_T(cx);
typedef struct { ORC_T(cx) a, b, c, d; } ORC_T(mat);

static inline ORC_T(cx) ORC_T(cmul)(ORC_T(cx) x, ORC_T(cx) y)
{
    ORC_T(cx) r;
    r.re = x.re * y.re - x.im * y.im;
    r.im = x.re * y.im + x.im * y.re;
    return r;
}

/* x * conj(y) */
static inline ORC_T(cx) ORC_T(cmulc)(ORC_T(cx) x, ORC_T(cx) y)
{
    ORC_T(cx) r;
    r.re = x.re * y.re + x.im * y.im;
    r.im = x.im * y.re - x.re * y.im;
    return r;
}

static inline ORC_T(cx) ORC_T(cadd)(ORC_T(cx) x, ORC_T(cx) y)
{
    ORC_T(cx) r; r.re = x.re + y.re; r.im = x.im + y.im; return r;
}

static inline ORC_T(mat) ORC_T(load_mat)(const REAL* p)
{
    ORC_T(mat) m;
    m.a.re = p[0]; m.a.im = p[1]; m.b.re = p[2]; m.b.im = p[3];
    m.c.re = p[4]; m.c.im = p[5]; m.d.re = p[6]; m.d.im = p[7];
    return m;
}

/*
 * J * B for the Hermitian brightness matrix
 * B = [[I+Q, U+iV], [U-iV, I-Q]]
 * (correlate/define_correlate_utils.h:36-39 builds B;
 *  math/define_multiply.h:74-87 multiplies by it).
 */
static inline ORC_T(mat) ORC_T(mul_brightness)(ORC_T(mat) J, REAL I, REAL Q,
        REAL U, REAL V)
{
    ORC_T(mat) r;
    ORC_T(cx) buv, buv_c;
    const REAL xx = I + Q, yy = I - Q;
    buv.re = U; buv.im = V;       /* B.b */
    buv_c.re = U; buv_c.im = -V;  /* B.c = conj(B.b) */
    r.a.re = J.a.re * xx; r.a.im = J.a.im * xx;
    r.a = ORC_T(cadd)(r.a, ORC_T(cmul)(J.b, buv_c));
    r.c.re = J.c.re * xx; r.c.im = J.c.im * xx;
    r.c = ORC_T(cadd)(r.c, ORC_T(cmul)(J.d, buv_c));
    r.b.re = J.b.re * yy; r.b.im = J.b.im * yy;
    r.b = ORC_T(cadd)(r.b, ORC_T(cmul)(J.a, buv));
    r.d.re = J.d.re * yy; r.d.im = J.d.im * yy;
    r.d = ORC_T(cadd)(r.d, ORC_T(cmul)(J.c, buv));
    return r;
}

/* M * N^H (math/define_multiply.h:54-67). */
static inline ORC_T(mat) ORC_T(mul_herm)(ORC_T(mat) M, ORC_T(mat) N)
{
    ORC_T(mat) r;
    r.a = ORC_T(cadd)(ORC_T(cmulc)(M.a, N.a), ORC_T(cmulc)(M.b, N.b));
    r.c = ORC_T(cadd)(ORC_T(cmulc)(M.c, N.a), ORC_T(cmulc)(M.d, N.b));
    r.b = ORC_T(cadd)(ORC_T(cmulc)(M.a, N.c), ORC_T(cmulc)(M.b, N.d));
    r.d = ORC_T(cadd)(ORC_T(cmulc)(M.c, N.c), ORC_T(cmulc)(M.d, N.d));
    return r;
}

/* sinc used for smearing (utility/oskar_kernel_macros.h:281). */
static inline REAL ORC_T(sinc)(REAL x)
{
    return x == (REAL)0 ? (REAL)1 : ORC_SIN(x) / x;
}

/*
 * Per-baseline terms: uu, vv, ww in wavelengths scaled by pi*frac_bandwidth,
 * the Gaussian quadratic-form terms and the uv length
 * (correlate/define_correlate_utils.h:5-13).
 */
typedef struct {
    REAL uu, vv, ww, uu2, vv2, uuvv, uv_len, du, dv, dw;
} ORC_T(bl);

static inline ORC_T(bl) ORC_T(baseline_terms)(int p, int q,
        const REAL* st_u, const REAL* st_v, const REAL* st_w,
        const REAL* st_x, const REAL* st_y, REAL inv_wavelength,
        REAL frac_bandwidth, int time_smearing, REAL time_int_sec,
        REAL gha0_rad, REAL dec0_rad)
{
    ORC_T(bl) t;
    REAL f;
    t.uu = (st_u[p] - st_u[q]) * inv_wavelength;
    t.vv = (st_v[p] - st_v[q]) * inv_wavelength;
    t.ww = (st_w[p] - st_w[q]) * inv_wavelength;
    t.uu2 = t.uu * t.uu;
    t.vv2 = t.vv * t.vv;
    t.uv_len = ORC_SQRT((REAL)(t.uu2 + t.vv2));
    t.uuvv = 2 * t.uu * t.vv;
    f = ((REAL) ORC_PI) * frac_bandwidth;
    t.uu *= f; t.vv *= f; t.ww *= f;
    t.du = t.dv = t.dw = 0;
    if (time_smearing)
    {
        /* Rotation of the baseline during the averaging time
         * (correlate/define_correlate_utils.h:15-27). */
        const REAL s_ha = ORC_SIN(gha0_rad), c_ha = ORC_COS(gha0_rad);
        const REAL s_dec = ORC_SIN(dec0_rad), c_dec = ORC_COS(dec0_rad);
        const REAL k = ((REAL) ORC_PI) * inv_wavelength;
        const REAL xx = (st_x[p] - st_x[q]) * k;
        const REAL yy = (st_y[p] - st_y[q]) * k;
        const REAL rot = ((REAL) ORC_OMEGA_EARTH) * time_int_sec;
        const REAL tmp = (xx * s_ha + yy * c_ha) * rot;
        t.du = (xx * c_ha - yy * s_ha) * rot;
        t.dv = tmp * s_dec;
        t.dw = -tmp * c_dec;
    }
    return t;
}

/* Smearing factor of one source on one baseline
 * (correlate/oskar_cross_correlate_omp.cpp:100-124). */
static inline REAL ORC_T(smearing)(const ORC_T(bl)* t, int i, int gaussian,
        int bw, int ts, const REAL* l, const REAL* m, const REAL* n,
        const REAL* a, const REAL* b, const REAL* c)
{
    REAL s = 1;
    if (gaussian)
    {
        const REAL e = a[i] * t->uu2 + b[i] * t->uuvv + c[i] * t->vv2;
        s = ORC_EXP((REAL) -e);
    }
    if (bw || ts)
    {
        const REAL ll = l[i], mm = m[i], nn = n[i] - (REAL)1;
        if (bw) s *= ORC_T(sinc)(t->uu * ll + t->vv * mm + t->ww * nn);
        if (ts) s *= ORC_T(sinc)(t->du * ll + t->dv * mm + t->dw * nn);
    }
    return s;
}

static inline int ORC_T(bl_index)(int num_st, int p, int q)
{
    return q * (num_st - 1) - (q - 1) * q / 2 + p - q - 1;
}

/*
 * Matrix cross-correlation: vis[bl] += sum_s smear * J_p B J_q^H.
 * Restates correlate/oskar_cross_correlate_omp.cpp:27-156 (kernel selection
 * by frac_bandwidth / time_int_sec as in XCORR_SELECT, :172-180). Single
 * precision uses Kahan summation as the reference does (:140-148).
 */
void ORC_FN(orc_xcorr_matrix)(int casa, int gaussian, int num_src,
        int num_st, int offset_out, const REAL* jones, const REAL* I,
        const REAL* Q, const REAL* U, const REAL* V, const REAL* l,
        const REAL* m, const REAL* n, const REAL* a, const REAL* b,
        const REAL* c, const REAL* st_u, const REAL* st_v, const REAL* st_w,
        const REAL* st_x, const REAL* st_y, REAL uv_min_lambda,
        REAL uv_max_lambda, REAL inv_wavelength, REAL frac_bandwidth,
        REAL time_int_sec, REAL gha0_rad, REAL dec0_rad, REAL* vis)
{
    const int bw = (frac_bandwidth != (REAL)0), ts = (time_int_sec != (REAL)0);
    int q;
#pragma omp parallel for schedule(dynamic, 1)
    for (q = 0; q < num_st; ++q)
    {
        int p;
        for (p = q + 1; p < num_st; ++p)
        {
            REAL sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            REAL guard[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            const int first = casa ? q : p, second = casa ? p : q;
            const REAL* jp = jones + 8 * (size_t) num_src * first;
            const REAL* jq = jones + 8 * (size_t) num_src * second;
            const ORC_T(bl) t = ORC_T(baseline_terms)(p, q, st_u, st_v, st_w,
                    st_x, st_y, inv_wavelength, frac_bandwidth, ts,
                    time_int_sec, gha0_rad, dec0_rad);
            int i, k;
            if (t.uv_len < uv_min_lambda || t.uv_len > uv_max_lambda)
                continue;
            for (i = 0; i < num_src; ++i)
            {
                const REAL s = ORC_T(smearing)(&t, i, gaussian, bw, ts,
                        l, m, n, a, b, c);
                const ORC_T(mat) mb = ORC_T(mul_brightness)(
                        ORC_T(load_mat)(jp + 8 * (size_t) i),
                        I[i], Q[i], U[i], V[i]);
                const ORC_T(mat) r = ORC_T(mul_herm)(mb,
                        ORC_T(load_mat)(jq + 8 * (size_t) i));
                const REAL term[8] = {r.a.re, r.a.im, r.b.re, r.b.im,
                        r.c.re, r.c.im, r.d.re, r.d.im};
                for (k = 0; k < 8; ++k)
                {
                    if (ORC_KAHAN)
                    {
                        const REAL y = term[k] * s - guard[k];
                        const REAL tt = sum[k] + y;
                        guard[k] = (tt - sum[k]) - y;
                        sum[k] = tt;
                    }
                    else sum[k] += term[k] * s;
                }
            }
            {
                REAL* out = vis + 8 * (size_t) (
                        ORC_T(bl_index)(num_st, p, q) + offset_out);
                for (k = 0; k < 8; ++k) out[k] += sum[k];
            }
        }
    }
}

/*
 * Scalar cross-correlation: vis[bl] += sum_s smear * I_s * J_p conj(J_q).
 * Restates the scalar CPU kernel (correlate/define_cross_correlate.h:157-187,
 * instantiated in correlate/src/oskar_cross_correlate_scalar_omp.cpp).
 */
void ORC_FN(orc_xcorr_scalar)(int casa, int gaussian, int num_src,
        int num_st, int offset_out, const REAL* jones, const REAL* I,
        const REAL* Q, const REAL* U, const REAL* V, const REAL* l,
        const REAL* m, const REAL* n, const REAL* a, const REAL* b,
        const REAL* c, const REAL* st_u, const REAL* st_v, const REAL* st_w,
        const REAL* st_x, const REAL* st_y, REAL uv_min_lambda,
        REAL uv_max_lambda, REAL inv_wavelength, REAL frac_bandwidth,
        REAL time_int_sec, REAL gha0_rad, REAL dec0_rad, REAL* vis)
{
    const int bw = (frac_bandwidth != (REAL)0), ts = (time_int_sec != (REAL)0);
    int q;
    (void) Q; (void) U; (void) V;
#pragma omp parallel for schedule(dynamic, 1)
    for (q = 0; q < num_st; ++q)
    {
        int p;
        for (p = q + 1; p < num_st; ++p)
        {
            REAL sre = 0, sim = 0;
            const int first = casa ? q : p, second = casa ? p : q;
            const REAL* jp = jones + 2 * (size_t) num_src * first;
            const REAL* jq = jones + 2 * (size_t) num_src * second;
            const ORC_T(bl) t = ORC_T(baseline_terms)(p, q, st_u, st_v, st_w,
                    st_x, st_y, inv_wavelength, frac_bandwidth, ts,
                    time_int_sec, gha0_rad, dec0_rad);
            int i;
            if (t.uv_len < uv_min_lambda || t.uv_len > uv_max_lambda)
                continue;
            for (i = 0; i < num_src; ++i)
            {
                const REAL s = ORC_T(smearing)(&t, i, gaussian, bw, ts,
                        l, m, n, a, b, c) * I[i];
                ORC_T(cx) x, y;
                x.re = jp[2 * i]; x.im = jp[2 * i + 1];
                y.re = jq[2 * i]; y.im = jq[2 * i + 1];
                x = ORC_T(cmulc)(x, y);
                sre += x.re * s;
                sim += x.im * s;
            }
            {
                REAL* out = vis + 2 * (size_t) (
                        ORC_T(bl_index)(num_st, p, q) + offset_out);
                out[0] += sre; out[1] += sim;
            }
        }
    }
}

/* Auto-correlation, matrix form (correlate/define_auto_correlate.h:36-57). */
void ORC_FN(orc_acorr_matrix)(int num_src, int num_st, int offset_out,
        const REAL* jones, const REAL* I, const REAL* Q, const REAL* U,
        const REAL* V, REAL* vis)
{
    int s;
#pragma omp parallel for
    for (s = 0; s < num_st; ++s)
    {
        REAL sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const REAL* js = jones + 8 * (size_t) num_src * s;
        int i, k;
        for (i = 0; i < num_src; ++i)
        {
            const ORC_T(mat) j = ORC_T(load_mat)(js + 8 * (size_t) i);
            const ORC_T(mat) r = ORC_T(mul_herm)(
                    ORC_T(mul_brightness)(j, I[i], Q[i], U[i], V[i]), j);
            sum[0] += r.a.re; sum[1] += r.a.im; sum[2] += r.b.re;
            sum[3] += r.b.im; sum[4] += r.c.re; sum[5] += r.c.im;
            sum[6] += r.d.re; sum[7] += r.d.im;
        }
        sum[1] = sum[7] = 0;
        for (k = 0; k < 8; ++k) vis[8 * (size_t) (s + offset_out) + k] += sum[k];
    }
}

/* Auto-correlation, scalar form (correlate/define_auto_correlate.h:84-101). */
void ORC_FN(orc_acorr_scalar)(int num_src, int num_st, int offset_out,
        const REAL* jones, const REAL* I, REAL* vis)
{
    int s;
#pragma omp parallel for
    for (s = 0; s < num_st; ++s)
    {
        REAL sum = 0;
        const REAL* js = jones + 2 * (size_t) num_src * s;
        int i;
        for (i = 0; i < num_src; ++i)
            sum += (js[2 * i] * js[2 * i] + js[2 * i + 1] * js[2 * i + 1])
                    * I[i];
        vis[2 * (size_t) (s + offset_out)] += sum;
    }
}

/*
 * Interferometer phase K[station][source] = exp(i * wavenumber *
 * (u l + v m + w (n - 1))), zero where the filter value is outside
 * (filter_min, filter_max]
 * (interferometer/define_evaluate_jones_K.h:56-70).
 */
void ORC_FN(orc_jones_k)(int num_src, const REAL* l, const REAL* m,
        const REAL* n, int num_st, const REAL* u, const REAL* v,
        const REAL* w, REAL wavenumber, const REAL* filter,
        REAL filter_min, REAL filter_max, int ignore_w, REAL* jones)
{
    int a;
#pragma omp parallel for
    for (a = 0; a < num_st; ++a)
    {
        int s;
        for (s = 0; s < num_src; ++s)
        {
            REAL re = 0, im = 0;
            if (filter[s] > filter_min && filter[s] <= filter_max)
            {
                REAL ph = u[a] * l[s] + v[a] * m[s];
                if (!ignore_w) ph += w[a] * (n[s] - (REAL)1);
                ph *= wavenumber;
                im = ORC_SIN(ph);
                re = ORC_COS(ph);
            }
            jones[2 * ((size_t) s + (size_t) num_src * a)] = re;
            jones[2 * ((size_t) s + (size_t) num_src * a) + 1] = im;
        }
    }
}

/* Element-wise products used by oskar_jones_join / oskar_mem_multiply
 * (mem/define_mem_multiply.h:14-89). */
void ORC_FN(orc_mem_mul_cc_c)(int n, const REAL* a, const REAL* b, REAL* c)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        ORC_T(cx) x, y, r;
        x.re = a[2 * i]; x.im = a[2 * i + 1];
        y.re = b[2 * i]; y.im = b[2 * i + 1];
        r = ORC_T(cmul)(x, y);
        c[2 * i] = r.re; c[2 * i + 1] = r.im;
    }
}

void ORC_FN(orc_mem_mul_cc_m)(int n, const REAL* a, const REAL* b, REAL* c)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        ORC_T(cx) x, y, r;
        x.re = a[2 * i]; x.im = a[2 * i + 1];
        y.re = b[2 * i]; y.im = b[2 * i + 1];
        r = ORC_T(cmul)(x, y);
        c[8 * i + 0] = r.re; c[8 * i + 1] = r.im;
        c[8 * i + 2] = 0; c[8 * i + 3] = 0;
        c[8 * i + 4] = 0; c[8 * i + 5] = 0;
        c[8 * i + 6] = r.re; c[8 * i + 7] = r.im;
    }
}

/* complex scalar (a) times matrix (b) */
void ORC_FN(orc_mem_mul_cm_m)(int n, const REAL* a, const REAL* b, REAL* c)
{
    int i, k;
    for (i = 0; i < n; ++i)
    {
        ORC_T(cx) s;
        s.re = a[2 * i]; s.im = a[2 * i + 1];
        for (k = 0; k < 4; ++k)
        {
            ORC_T(cx) x, r;
            x.re = b[8 * i + 2 * k]; x.im = b[8 * i + 2 * k + 1];
            r = ORC_T(cmul)(x, s);
            c[8 * i + 2 * k] = r.re; c[8 * i + 2 * k + 1] = r.im;
        }
    }
}

/* matrix (a) times complex scalar (b) */
void ORC_FN(orc_mem_mul_mc_m)(int n, const REAL* a, const REAL* b, REAL* c)
{
    int i, k;
    for (i = 0; i < n; ++i)
    {
        ORC_T(cx) s;
        s.re = b[2 * i]; s.im = b[2 * i + 1];
        for (k = 0; k < 4; ++k)
        {
            ORC_T(cx) x, r;
            x.re = a[8 * i + 2 * k]; x.im = a[8 * i + 2 * k + 1];
            r = ORC_T(cmul)(x, s);
            c[8 * i + 2 * k] = r.re; c[8 * i + 2 * k + 1] = r.im;
        }
    }
}

/* matrix (a) times matrix (b) */
void ORC_FN(orc_mem_mul_mm_m)(int n, const REAL* a, const REAL* b, REAL* c)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        const ORC_T(mat) x = ORC_T(load_mat)(a + 8 * (size_t) i);
        const ORC_T(mat) y = ORC_T(load_mat)(b + 8 * (size_t) i);
        ORC_T(mat) r;
        r.a = ORC_T(cadd)(ORC_T(cmul)(x.a, y.a), ORC_T(cmul)(x.b, y.c));
        r.c = ORC_T(cadd)(ORC_T(cmul)(x.c, y.a), ORC_T(cmul)(x.d, y.c));
        r.b = ORC_T(cadd)(ORC_T(cmul)(x.a, y.b), ORC_T(cmul)(x.b, y.d));
        r.d = ORC_T(cadd)(ORC_T(cmul)(x.c, y.b), ORC_T(cmul)(x.d, y.d));
        c[8 * i + 0] = r.a.re; c[8 * i + 1] = r.a.im;
        c[8 * i + 2] = r.b.re; c[8 * i + 3] = r.b.im;
        c[8 * i + 4] = r.c.re; c[8 * i + 5] = r.c.im;
        c[8 * i + 6] = r.d.re; c[8 * i + 7] = r.d.im;
    }
}

/*
 * Weighted DFT of element signals to output directions.
 *   out[d] = norm * sum_e w_e * exp(i k (x_e X_d + y_e Y_d [+ z_e Z_d]))
 *                 * data[idx_e][d]
 * matrix = 0: complex data [num_types][num_out], output [num_out];
 * matrix = 1: data [num_types][num_out][4] (xx, xy, yx, yy), only the pairs
 * selected by eval_x / eval_y are written.
 * Restates math/define_dftw_c2c.h:79-106 and math/define_dftw_m2m.h:109-167.
 */
void ORC_FN(orc_dftw)(int matrix, int is_3d, int num_in, REAL wavenumber,
        const REAL* weights_in, const REAL* x_in, const REAL* y_in,
        const REAL* z_in, int offset_coord_out, int num_out,
        const REAL* x_out, const REAL* y_out, const REAL* z_out,
        const int* data_idx, const REAL* data, int eval_x, int eval_y,
        int offset_out, REAL* output, REAL norm_factor)
{
    int d;
#pragma omp parallel for
    for (d = 0; d < num_out; ++d)
    {
        REAL acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        const REAL xo = wavenumber * x_out[d + offset_coord_out];
        const REAL yo = wavenumber * y_out[d + offset_coord_out];
        const REAL zo = is_3d ? wavenumber * z_out[d + offset_coord_out] : 0;
        int e, k;
        for (e = 0; e < num_in; ++e)
        {
            REAL ph = xo * x_in[e] + yo * y_in[e];
            REAL re, im, cre;
            const int src = data_idx ? data_idx[e] : e;
            if (is_3d) ph += zo * z_in[e];
            im = ORC_SIN(ph);
            re = ORC_COS(ph);
            /* phasor times weight */
            cre = re;
            re = re * weights_in[2 * e] - weights_in[2 * e + 1] * im;
            im = im * weights_in[2 * e] + weights_in[2 * e + 1] * cre;
            if (!matrix)
            {
                const REAL* in = data + 2 * ((size_t) src * num_out + d);
                acc[0] += in[0] * re - in[1] * im;
                acc[1] += in[1] * re + in[0] * im;
            }
            else
            {
                const REAL* in = data + 8 * ((size_t) src * num_out + d);
                const int k0 = eval_x ? 0 : 2, k1 = eval_y ? 4 : 2;
                for (k = k0; k < k1; ++k)
                {
                    acc[2 * k] += in[2 * k] * re - in[2 * k + 1] * im;
                    acc[2 * k + 1] += in[2 * k + 1] * re + in[2 * k] * im;
                }
            }
        }
        if (!matrix)
        {
            output[2 * ((size_t) d + offset_out)] = acc[0] * norm_factor;
            output[2 * ((size_t) d + offset_out) + 1] = acc[1] * norm_factor;
        }
        else
        {
            REAL* o = output + 8 * ((size_t) d + offset_out);
            const int k0 = eval_x ? 0 : 2, k1 = eval_y ? 4 : 2;
            for (k = k0; k < k1; ++k)
            {
                o[2 * k] = acc[2 * k] * norm_factor;
                o[2 * k + 1] = acc[2 * k + 1] * norm_factor;
            }
        }
    }
}

/* Beamforming weights w_e = exp(-i k (x x1 + y y1 + z z1 + cable_e))
 * (telescope/station/define_evaluate_element_weights_dft.h:3-16). */
void ORC_FN(orc_element_weights_dft)(int n, const REAL* x, const REAL* y,
        const REAL* z, const REAL* cable_length_error, REAL wavenumber,
        REAL x1, REAL y1, REAL z1, REAL* weights)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        const REAL p = wavenumber * (x[i] * x1 + y[i] * y1 + z[i] * z1 +
                cable_length_error[i]);
        weights[2 * i] = ORC_COS(-p);
        weights[2 * i + 1] = ORC_SIN(-p);
    }
}

/* Station ECEF offsets to (u, v, w) at hour angle ha0
 * (convert/define_convert_ecef_to_station_uvw.h:3-29). */
void ORC_FN(orc_ecef_to_station_uvw)(int n, const REAL* x, const REAL* y,
        const REAL* z, REAL sin_ha0, REAL cos_ha0, REAL sin_dec0,
        REAL cos_dec0, int ignore_w, int offset_out, REAL* u, REAL* v,
        REAL* w)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        const REAL xx = x[i], yy = y[i], zz = z[i];
        const REAL t = xx * cos_ha0 - yy * sin_ha0;
        u[i + offset_out] = xx * sin_ha0 + yy * cos_ha0;
        v[i + offset_out] = zz * cos_dec0 - t * sin_dec0;
        w[i + offset_out] = ignore_w ? (REAL)0 : zz * sin_dec0 + t * cos_dec0;
    }
}

/* ENU direction cosines to element-frame (theta, phi_x, phi_y), phi wrapped
 * into [0, 2 pi), with an optional extra point at the pole carrying the
 * unwrapped phase offsets
 * (convert/define_convert_enu_directions_to_theta_phi.h:3-31). */
void ORC_FN(orc_enu_to_theta_phi)(int off_in, int num, const REAL* x,
        const REAL* y, const REAL* z, int extra_point_at_pole, REAL dphi1,
        REAL dphi2, REAL* theta, REAL* phi1, REAL* phi2)
{
    const REAL twopi = 2 * (REAL) ORC_PI;
    int i;
    for (i = 0; i < num; ++i)
    {
        const REAL xx = x[i + off_in], yy = y[i + off_in], zz = z[i + off_in];
        const REAL p0 = ORC_ATAN2(yy, xx);
        REAL p1 = ORC_FMOD(p0 + dphi1, twopi);
        REAL p2 = ORC_FMOD(p0 + dphi2, twopi);
        if (p1 < 0) p1 += twopi;
        if (p2 < 0) p2 += twopi;
        theta[i] = ORC_ATAN2(ORC_SQRT(xx * xx + yy * yy), zz);
        phi1[i] = p1;
        phi2[i] = p2;
    }
    if (extra_point_at_pole)
    {
        theta[num] = 0;
        phi1[num] = dphi1;
        phi2[num] = dphi2;
    }
}

/* Far field of one half-wave-style dipole of electrical half-length kL
 * along the direction phi (define_evaluate_dipole_pattern.h:3-15). */
static void ORC_T(dipole)(REAL kL, REAL cos_kL, REAL sin_th, REAL cos_th,
        REAL phi, REAL* e_theta, REAL* e_phi)
{
    const REAL sp = ORC_SIN(phi), cp = ORC_COS(phi);
    const REAL denom = 1 + cp * cp * (cos_th * cos_th - 1);
    REAL t;
    if (denom == 0)
    {
        *e_theta = *e_phi = 0;
        return;
    }
    t = (ORC_COS(kL * cp * sin_th) - cos_kL) / denom;
    *e_theta = -cp * cos_th * t;
    *e_phi = sp * t;
}

/* Polarised dipole pattern {x_theta, x_phi, y_theta, y_phi}, X and Y rows
 * swapped if swap_xy (define_evaluate_dipole_pattern.h:17-48). */
void ORC_FN(orc_dipole_pattern)(int n, const REAL* theta, const REAL* phi_x,
        const REAL* phi_y, REAL kL, REAL cos_kL, int swap_xy, int offset_out,
        REAL* pattern)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        REAL xt, xp, yt, yp;
        const REAL st = ORC_SIN(theta[i]), ct = ORC_COS(theta[i]);
        REAL* o = pattern + 8 * ((size_t) i + offset_out);
        ORC_T(dipole)(kL, cos_kL, st, ct, phi_x[i], &xt, &xp);
        ORC_T(dipole)(kL, cos_kL, st, ct, phi_y[i], &yt, &yp);
        o[0] = swap_xy ? yt : xt;
        o[2] = swap_xy ? yp : xp;
        o[4] = swap_xy ? xt : yt;
        o[6] = swap_xy ? xp : yp;
        o[1] = o[3] = o[5] = o[7] = 0;
    }
}

/* Scales matrices [offset, offset + n), except the one at idx, by
 * 1 / sqrt(|M_idx|_F^2 / 2) (mem/define_mem_normalise.h:31-51). */
void ORC_FN(orc_mem_normalise_matrix)(int offset, int n, REAL* a, int idx)
{
    const REAL* v = a + 8 * (size_t) idx;
    REAL amp = 0, scal;
    int j, k;
    for (k = 0; k < 8; ++k) amp += v[k] * v[k];
    scal = 1 / ORC_SQRT(amp / 2);
    for (j = offset; j < offset + n; ++j)
    {
        if (j == idx) continue;
        for (k = 0; k < 8; ++k) a[8 * (size_t) j + k] *= scal;
    }
}

/* Zeroes matrices whose direction has z < 0
 * (telescope/station/define_blank_below_horizon.h:15-29). */
void ORC_FN(orc_blank_below_horizon)(int off_mask, int n, const REAL* mask,
        int off_out, REAL* jones)
{
    int i, k;
    for (i = 0; i < n; ++i)
        if (mask[i + off_mask] < 0)
            for (k = 0; k < 8; ++k) jones[8 * ((size_t) i + off_out) + k] = 0;
}

/* Parallactic-angle rotation R for each source as seen from a station at
 * latitude lat and local sidereal time lst
 * (interferometer/define_evaluate_jones_R.h:3-29). */
void ORC_FN(orc_jones_r)(int num_sources, const REAL* ra, const REAL* dec,
        REAL cos_lat, REAL sin_lat, REAL lst_rad, int offset_out, REAL* jones)
{
    int i;
    for (i = 0; i < num_sources; ++i)
    {
        const REAL ha = lst_rad - ra[i];
        const REAL sh = ORC_SIN(ha), ch = ORC_COS(ha);
        const REAL sd = ORC_SIN(dec[i]), cd = ORC_COS(dec[i]);
        const REAL q = ORC_ATAN2(cos_lat * sh, sin_lat * cd - cos_lat * sd * ch);
        const REAL sq = ORC_SIN(q), cq = ORC_COS(q);
        REAL* o = jones + 8 * ((size_t) i + offset_out);
        o[0] = cq; o[2] = -sq; o[4] = sq; o[6] = cq;
        o[1] = o[3] = o[5] = o[7] = 0;
    }
}

/* Aperture-array station beam for one station with a single element type
 * (dipoles, common orientation) and one feed set, composed exactly as the
 * reference composes it:
 *  - oskar_station_beam (telescope/station/src/oskar_station_beam.c:84-91,
 *    107-135, 178-182): zero beam if the pointing is below the horizon; the
 *    normalisation direction appended as an extra point and the beam
 *    divided by its amplitude at the end;
 *  - oskar_evaluate_station_beam_aperture_array
 *    (telescope/station/src/oskar_evaluate_station_beam_aperture_array.c:
 *    150-240): element pattern (oskar_element_evaluate.c:76-80, 134-138,
 *    153-157, orientation_x offset by pi/2), weights from the measured
 *    element positions (oskar_station_evaluate_element_weights.c:25-31),
 *    weighted DFT over the true positions, horizon blanking.
 * Scalars that the reference derives in double (wavenumber, kL, delta phi)
 * are derived in double here too, then rounded to REAL. */
void ORC_FN(orc_station_beam_aa_types)(int num_el, int num_feeds,
        const REAL* x,
        const REAL* y, const REAL* z, const REAL* x_meas, const REAL* y_meas,
        const REAL* z_meas, const REAL* cable, const REAL* weight_factors,
        int num_types, const int* element_type,
        const double* dipole_length_per_type, const int* kind_per_type,
        const int* taper_per_type, const double* taper_param_per_type,
        const double* orientation_x_per_type,
        const double* orientation_y_per_type, int norm_element,
        int norm_array, int norm_final, int swap_xy, int scalar, int is_3d,
        double frequency_hz, double bx, double by, double bz, double nx,
        double ny, double nz, int num_dir, const REAL* dx, const REAL* dy,
        const REAL* dz, REAL* beam)
{
    const double c0 = 299792458.0;
    const int np = num_dir + (norm_final ? 1 : 0);
    const int npe = np + (norm_element ? 1 : 0);
    const double wavenumber = 2.0 * ORC_PI * frequency_hz / c0;
    REAL *X, *Y, *Z, *theta, *phi1, *phi2, *signal, *pattern, *w, *out;
    int* types;
    int i, t, f;
    if (bz < 0)
    {
        for (i = 0; i < 8 * num_dir; ++i) beam[i] = 0;
        return;
    }
    X = (REAL*) malloc(sizeof(REAL) * np);
    Y = (REAL*) malloc(sizeof(REAL) * np);
    Z = (REAL*) malloc(sizeof(REAL) * np);
    theta = (REAL*) malloc(sizeof(REAL) * npe);
    phi1 = (REAL*) malloc(sizeof(REAL) * npe);
    phi2 = (REAL*) malloc(sizeof(REAL) * npe);
    signal = (REAL*) calloc((size_t) 8 * np * num_types, sizeof(REAL));
    pattern = (REAL*) calloc((size_t) 8 * npe, sizeof(REAL));
    out = (REAL*) calloc((size_t) 8 * np, sizeof(REAL));
    w = (REAL*) malloc(sizeof(REAL) * 2 * num_el);
    types = (int*) calloc((size_t) num_el, sizeof(int));
    if (element_type)
        for (i = 0; i < num_el; ++i) types[i] = element_type[i];
    for (i = 0; i < num_dir; ++i)
    {
        X[i] = dx[i]; Y[i] = dy[i]; Z[i] = dz[i];
    }
    if (norm_final)
    {
        X[num_dir] = (REAL) nx; Y[num_dir] = (REAL) ny; Z[num_dir] = (REAL) nz;
    }
    /* one element pattern per type (oskar_evaluate_station_beam_aperture_
     * array.c:158-202: per element type, or per element when orientations
     * differ), each with its own orientation and normalised at its own
     * pole */
    for (t = 0; t < num_types; ++t)
    {
        const double kL = dipole_length_per_type[t] *
                (ORC_PI * frequency_hz / c0);
        const double dphi1 =
                ORC_PI / 2 - (orientation_x_per_type[t] + ORC_PI / 2);
        const double dphi2 = ORC_PI / 2 - orientation_y_per_type[t];
        ORC_FN(orc_enu_to_theta_phi)(0, np, X, Y, Z, norm_element,
                (REAL) dphi1, (REAL) dphi2, theta, phi1, phi2);
        if (kind_per_type && kind_per_type[t] == 1)
        {
            /* isotropic: the identity (oskar_element_evaluate.c:82-87) */
            for (i = 0; i < npe; ++i)
            {
                int k;
                for (k = 0; k < 8; ++k) pattern[8 * i + k] = 0;
                pattern[8 * i] = pattern[8 * i + 6] = 1;
            }
        }
        else
            ORC_FN(orc_dipole_pattern)(npe, theta, phi1, phi2, (REAL) kL,
                    (REAL) cos(kL), swap_xy, 0, pattern);
        if (norm_element)
            ORC_FN(orc_mem_normalise_matrix)(0, np, pattern, np);
        /* element taper after the normalisation (oskar_element_evaluate.c:
         * 159-174; define_apply_element_taper_{cosine,gaussian}.h) */
        if (taper_per_type && taper_per_type[t] != 0)
            for (i = 0; i < np; ++i)
            {
                int k;
                REAL fac;
                if (taper_per_type[t] == 1)
                    fac = (REAL) pow((REAL) cos(theta[i]),
                            (REAL) taper_param_per_type[t]);
                else
                {
                    const double fwhm = taper_param_per_type[t];
                    const REAL inv_2sigma_sq = (REAL)
                            (4.0 * log(2.0) / (fwhm * fwhm));
                    REAL th2 = theta[i];
                    th2 *= th2;
                    fac = ORC_EXP(-th2 * inv_2sigma_sq);
                }
                for (k = 0; k < 8; ++k) pattern[8 * i + k] *= fac;
            }
        for (i = 0; i < 8 * np; ++i)
            signal[(size_t) 8 * np * t + i] = pattern[i];
    }
    /* per feed: weights from that feed's measured positions, cable errors
     * and factors, then the weighted DFT over its true positions into the
     * feed's rows (oskar_evaluate_station_beam_aperture_array.c:208-223;
     * element arrays are [feed][element]) */
    for (f = 0; f < num_feeds; ++f)
    {
        const size_t o = (size_t) f * num_el;
        const REAL* xm = x_meas ? x_meas + o : x + o;
        const REAL* ym = y_meas ? y_meas + o : y + o;
        const REAL* zm = z_meas ? z_meas + o : z + o;
        ORC_FN(orc_element_weights_dft)(num_el, xm, ym, zm, cable + o,
                (REAL) wavenumber, (REAL) bx, (REAL) by, (REAL) bz, w);
        /* element errors, gains, apodisation: weights *= factor
         * (oskar_station_evaluate_element_weights.c:33-64) */
        if (weight_factors)
            for (i = 0; i < num_el; ++i)
            {
                ORC_T(cx) a = {w[2 * i], w[2 * i + 1]};
                const ORC_T(cx) fc = {weight_factors[2 * (o + i)],
                        weight_factors[2 * (o + i) + 1]};
                a = ORC_T(cmul)(a, fc);
                w[2 * i] = a.re;
                w[2 * i + 1] = a.im;
            }
        ORC_FN(orc_dftw)(1, is_3d, num_el, (REAL) wavenumber, w, x + o,
                y + o, z + o, 0, np, X, Y, is_3d ? Z : 0, types, signal,
                f == 0 || num_feeds == 1, f == 1 || num_feeds == 1, 0, out,
                norm_array ? (REAL) (1.0 / num_el) : (REAL) 1);
    }
    if (scalar)
    {
        /* scalar response: the pattern amplitude sqrt(sum of the four
         * real terms squared / 2) (define_evaluate_dipole_pattern.h:51-75;
         * it commutes with the pole normalisation and the taper), a
         * complex DFT, horizon blanking, and division by the magnitude in
         * the normalisation direction (define_mem_normalise.h:13-29) */
        REAL* ssig = (REAL*) calloc((size_t) 2 * np * num_types,
                sizeof(REAL));
        for (i = 0; i < np * num_types; ++i)
        {
            const REAL* m = signal + 8 * (size_t) i;
            ssig[2 * i] = ORC_SQRT((m[0] * m[0] + m[2] * m[2] +
                    m[4] * m[4] + m[6] * m[6]) / 2);
        }
        for (i = 0; i < 2 * np; ++i) out[i] = 0;
        for (f = 0; f < num_feeds; ++f)
        {
            const size_t o = (size_t) f * num_el;
            const REAL* xm = x_meas ? x_meas + o : x + o;
            const REAL* ym = y_meas ? y_meas + o : y + o;
            const REAL* zm = z_meas ? z_meas + o : z + o;
            ORC_FN(orc_element_weights_dft)(num_el, xm, ym, zm, cable + o,
                    (REAL) wavenumber, (REAL) bx, (REAL) by, (REAL) bz, w);
            if (weight_factors)
                for (i = 0; i < num_el; ++i)
                {
                    ORC_T(cx) a = {w[2 * i], w[2 * i + 1]};
                    const ORC_T(cx) fc = {weight_factors[2 * (o + i)],
                            weight_factors[2 * (o + i) + 1]};
                    a = ORC_T(cmul)(a, fc);
                    w[2 * i] = a.re;
                    w[2 * i + 1] = a.im;
                }
            ORC_FN(orc_dftw)(0, is_3d, num_el, (REAL) wavenumber, w, x + o,
                    y + o, z + o, 0, np, X, Y, is_3d ? Z : 0, types, ssig,
                    1, 1, 0, out,
                    norm_array ? (REAL) (1.0 / num_el) : (REAL) 1);
        }
        for (i = 0; i < np; ++i)
            if (Z[i] < 0) out[2 * i] = out[2 * i + 1] = 0;
        if (norm_final)
        {
            const REAL* v = out + 2 * (size_t) (np - 1);
            const REAL scal = 1 / ORC_SQRT(v[0] * v[0] + v[1] * v[1]);
            for (i = 0; i < np - 1; ++i)
            {
                out[2 * i] *= scal;
                out[2 * i + 1] *= scal;
            }
        }
        for (i = 0; i < 2 * num_dir; ++i) beam[i] = out[i];
        free(ssig);
    }
    else
    {
        ORC_FN(orc_blank_below_horizon)(0, np, Z, 0, out);
        if (norm_final) ORC_FN(orc_mem_normalise_matrix)(0, np, out, np - 1);
        for (i = 0; i < 8 * num_dir; ++i) beam[i] = out[i];
    }
    free(X); free(Y); free(Z); free(theta); free(phi1); free(phi2);
    free(signal); free(pattern); free(out); free(w); free(types);
}

void ORC_FN(orc_station_beam_aa_weighted)(int num_el, const REAL* x,
        const REAL* y, const REAL* z, const REAL* x_meas, const REAL* y_meas,
        const REAL* z_meas, const REAL* cable, const REAL* weight_factors,
        double orientation_x_rad, double orientation_y_rad,
        double dipole_length_m, int norm_element, int norm_array,
        int norm_final, int swap_xy, int is_3d, double frequency_hz,
        double bx, double by, double bz, double nx, double ny, double nz,
        int num_dir, const REAL* dx, const REAL* dy, const REAL* dz,
        REAL* beam)
{
    ORC_FN(orc_station_beam_aa_types)(num_el, 1, x, y, z, x_meas, y_meas,
            z_meas, cable, weight_factors, 1, 0, &dipole_length_m, 0, 0, 0,
            &orientation_x_rad, &orientation_y_rad, norm_element, norm_array,
            norm_final, swap_xy, 0, is_3d, frequency_hz, bx, by, bz, nx, ny, nz,
            num_dir, dx, dy, dz, beam);
}

void ORC_FN(orc_station_beam_aa)(int num_el, const REAL* x, const REAL* y,
        const REAL* z, const REAL* x_meas, const REAL* y_meas,
        const REAL* z_meas, const REAL* cable, double orientation_x_rad,
        double orientation_y_rad, double dipole_length_m, int norm_element,
        int norm_array, int norm_final, int swap_xy, int is_3d,
        double frequency_hz, double bx, double by, double bz, double nx,
        double ny, double nz, int num_dir, const REAL* dx, const REAL* dy,
        const REAL* dz, REAL* beam)
{
    ORC_FN(orc_station_beam_aa_weighted)(num_el, x, y, z, x_meas, y_meas,
            z_meas, cable, 0, orientation_x_rad, orientation_y_rad,
            dipole_length_m, norm_element, norm_array, norm_final, swap_xy,
            is_3d, frequency_hz, bx, by, bz, nx, ny, nz, num_dir, dx, dy, dz,
            beam);
}

/* Relative direction cosines of (lon, lat) about (lon0, lat0)
 * (convert/define_convert_lon_lat_to_relative_directions.h:3-19); n is
 * skipped when NULL. */
void ORC_FN(orc_lon_lat_to_relative_directions)(int num, const REAL* lon,
        const REAL* lat, REAL lon0, REAL cos_lat0, REAL sin_lat0, REAL* l,
        REAL* m, REAL* n)
{
    int i;
    for (i = 0; i < num; ++i)
    {
        const REAL dl = lon[i] - lon0;
        const REAL sl = ORC_SIN(dl), cl = ORC_COS(dl);
        const REAL sb = ORC_SIN(lat[i]), cb = ORC_COS(lat[i]);
        l[i] = cb * sl;
        m[i] = cos_lat0 * sb - sin_lat0 * cb * cl;
        if (n) n[i] = sin_lat0 * sb + cos_lat0 * cb * cl;
    }
}

/* Apparent (RA, Dec) to the ENU direction cosines of a station at local
 * sidereal time lst and latitude lat
 * (convert/define_convert_apparent_ra_dec_to_enu_directions.h:3-30). */
void ORC_FN(orc_ra_dec_to_enu_directions)(int num, const REAL* ra,
        const REAL* dec, REAL lst, REAL sin_lat, REAL cos_lat, int offset_out,
        REAL* x, REAL* y, REAL* z)
{
    int i;
    for (i = 0; i < num; ++i)
    {
        const REAL ha = lst - ra[i];
        const REAL sh = ORC_SIN(ha), ch = ORC_COS(ha);
        const REAL sd = ORC_SIN(dec[i]), cd = ORC_COS(dec[i]);
        x[i + offset_out] = -cd * sh;
        y[i + offset_out] = cos_lat * sd - sin_lat * cd * ch;
        z[i + offset_out] = sin_lat * sd + cos_lat * cd * ch;
    }
}

/* mask |= (l l_mul + m m_mul + n n_mul > 0): the source is above a
 * station's horizon (sky/define_update_horizon_mask.h:3-12). */
void ORC_FN(orc_update_horizon_mask)(int num, const REAL* l, const REAL* m,
        const REAL* n, REAL l_mul, REAL m_mul, REAL n_mul, int* mask)
{
    int i;
    for (i = 0; i < num; ++i)
        mask[i] |= ((l[i] * l_mul + m[i] * m_mul + n[i] * n_mul) > 0);
}

/* Baseline (uu, vv, ww) = station 2 - station 1 for every pair s1 < s2,
 * negated in the CASA convention
 * (convert/define_convert_station_uvw_to_baseline_uvw.h:3-20). */
void ORC_FN(orc_station_uvw_to_baseline_uvw)(int casa, int num,
        int offset_in, const REAL* u, const REAL* v, const REAL* w,
        int offset_out, REAL* uu, REAL* vv, REAL* ww)
{
    const REAL f = casa ? -1 : 1;
    int s1, s2;
    for (s1 = 0; s1 < num; ++s1)
        for (s2 = s1 + 1; s2 < num; ++s2)
        {
            const int b = s1 * (num - 1) - (s1 - 1) * s1 / 2 + s2 - s1 - 1 +
                    offset_out;
            uu[b] = f * (u[s2 + offset_in] - u[s1 + offset_in]);
            vv[b] = f * (v[s2 + offset_in] - v[s1 + offset_in]);
            ww[b] = f * (w[s2 + offset_in] - w[s1 + offset_in]);
        }
}

/* ---- Sky flux scaling with frequency ----
 * The sky table is column-major: column k of source s at
 * table[capacity * k + s]; columns of one type are adjacent, in index order.
 * num_valid[s * 20 + type] counts the columns of each type that hold data
 * for source s. Type numbers follow the reference's column enumeration
 * (sky/oskar_sky_enum.h:14-35): I 3, Q 4, U 5, V 6, reference frequency 7,
 * spectral index 8, rotation measure 9, linear-index flag 13, polarisation
 * angle 14, polarisation fraction 15, reference wavelength 16, spectral
 * curvature 17, line width 18, frequency increment 19; 20 types in all.
 * A column index outside [0, num_columns) reads as 0 (the reference reads
 * past its table there). */
#ifndef ORC_SKY_ENUM_
#define ORC_SKY_ENUM_
enum { ORC_SKY_I = 3, ORC_SKY_Q = 4, ORC_SKY_U = 5, ORC_SKY_V = 6,
    ORC_SKY_REF_HZ = 7, ORC_SKY_SPX = 8, ORC_SKY_RM = 9, ORC_SKY_LIN_SI = 13,
    ORC_SKY_POLA = 14, ORC_SKY_POLF = 15, ORC_SKY_REF_WAVE = 16,
    ORC_SKY_CURV = 17, ORC_SKY_LINE_WIDTH = 18, ORC_SKY_INC_HZ = 19,
    ORC_SKY_NUM_TYPES = 20 };
#define ORC_C0_M_PER_S 299792458
/* slots of the column table below */
enum { ORC_CI = 0, ORC_CQ, ORC_CU, ORC_CV, ORC_CREF, ORC_CLIN, ORC_CSPX,
    ORC_CRM, ORC_CPOLF, ORC_CPOLA, ORC_CREFW, ORC_CCURV, ORC_CLW, ORC_CINC };
#endif

typedef struct
{
    const REAL* table;
    int capacity, num_columns;
    /* first column of: I Q U V ref_hz lin_si spx rm polf pola ref_wave curv
     * line_width inc_hz */
    int col[14];
} ORC_T(sky);


static REAL ORC_T(sky_at)(const ORC_T(sky)* k, int column, int s)
{
    if (column < 0 || column >= k->num_columns) return 0;
    return k->table[(size_t) k->capacity * column + s];
}

static REAL ORC_T(nan0)(REAL x) { return x != x ? (REAL) 0 : x; }

/* Stokes I of source s at freq_hz, given its value i_in at freq0_hz
 * (sky/define_sky_scale_flux_with_frequency.h:5-86): a sum of Gaussian line
 * profiles when line widths are given; the value unchanged when several I
 * columns are given; a curved power law (Callingham et al. 2017, eq. 2)
 * when a curvature is given; else the logarithmic spectral-index polynomial
 * (the default) or the linear one, both by Horner's rule. NaN coefficients
 * count as 0. Math in double, as the reference's C build computes it. */
static REAL ORC_T(stokes_i_at)(const ORC_T(sky)* k, const int* nv, int s,
        REAL i_in, REAL freq_hz, REAL freq0_hz)
{
    int c;
    const int n_i = nv[ORC_SKY_I], n_lw = nv[ORC_SKY_LINE_WIDTH];
    const int n_spx = nv[ORC_SKY_SPX];
    if (n_lw > 0)
    {
        const int n_ref = nv[ORC_SKY_REF_HZ];
        const REAL inc = nv[ORC_SKY_INC_HZ] > 0 ?
                ORC_T(sky_at)(k, k->col[ORC_CINC], s) : (REAL) 0;
        REAL sum = 0;
        for (c = 0; c < n_i; ++c)
        {
            const REAL amp = ORC_T(sky_at)(k, k->col[ORC_CI] + c, s);
            const REAL ref = c < n_ref ?
                    ORC_T(sky_at)(k, k->col[ORC_CREF] + c, s) :
                    ORC_T(sky_at)(k, k->col[ORC_CREF], s) + c * inc;
            const REAL sigma = ORC_T(sky_at)(k,
                    k->col[ORC_CLW] + (c < n_lw ? c : 0), s);
            const REAL x = freq_hz - ref;
            sum += amp * exp(-(x * x) / (2 * sigma * sigma));
        }
        return sum;
    }
    if (n_i > 1) return i_in;
    if (nv[ORC_SKY_CURV] > 0)
    {
        const REAL spx = n_spx > 0 ?
                ORC_T(nan0)(ORC_T(sky_at)(k, k->col[ORC_CSPX], s)) : 0;
        const REAL curv_coef = ORC_T(nan0)(
                ORC_T(sky_at)(k, k->col[ORC_CCURV], s));
        const REAL ratio = freq_hz / freq0_hz;
        const REAL lr = (REAL) log(ratio);
        const REAL curv = (REAL) exp(curv_coef * (lr * lr));
        return (REAL) (i_in * curv * pow(ratio, spx));
    }
    {
        const REAL lin = nv[ORC_SKY_LIN_SI] > 0 ?
                ORC_T(sky_at)(k, k->col[ORC_CLIN], s) : (REAL) 0;
        REAL acc = 0;
        if (lin == (REAL) 0)
        {
            const REAL base = (REAL) log10(freq_hz / freq0_hz);
            for (c = n_spx - 1; c >= 0; --c)
                acc = base * acc + ORC_T(nan0)(
                        ORC_T(sky_at)(k, k->col[ORC_CSPX] + c, s));
            return (REAL) (i_in * pow((REAL) 10, base * acc));
        }
        {
            const REAL base = freq_hz / freq0_hz - (REAL) 1;
            for (c = n_spx - 1; c >= 0; --c)
                acc = base * acc + ORC_T(nan0)(
                        ORC_T(sky_at)(k, k->col[ORC_CSPX] + c, s));
            return i_in + base * acc;
        }
    }
}

/* Scaled I, Q, U, V of every source at freq_hz
 * (sky/define_sky_scale_flux_with_frequency.h:89-253): the reference
 * channel nearest freq_hz, its Stokes values, Q and U from polarisation
 * angle and fraction where only those are given, then spectral scaling of
 * I (Q, U, V follow I's ratio) or, with a rotation measure, Faraday
 * rotation of the polarisation angle. Column arguments in the reference
 * kernel's order. */
void ORC_FN(orc_sky_scale_flux)(int num_sources, int capacity,
        int num_columns, REAL freq_hz, const REAL* table,
        const int* num_valid, int col_i, int col_q, int col_u, int col_v,
        int col_ref_freq, int col_lin_sp_index, int col_sp_index,
        int col_rot_meas, int col_pol_frac, int col_pol_ang,
        int col_ref_wavelength, int col_sp_curvature, int col_line_width,
        int col_freq_inc, REAL* out_i, REAL* out_q, REAL* out_u,
        REAL* out_v)
{
    ORC_T(sky) k;
    int s;
    k.table = table;
    k.capacity = capacity;
    k.num_columns = num_columns;
    k.col[ORC_CI] = col_i; k.col[ORC_CQ] = col_q; k.col[ORC_CU] = col_u;
    k.col[ORC_CV] = col_v; k.col[ORC_CREF] = col_ref_freq;
    k.col[ORC_CLIN] = col_lin_sp_index; k.col[ORC_CSPX] = col_sp_index;
    k.col[ORC_CRM] = col_rot_meas; k.col[ORC_CPOLF] = col_pol_frac;
    k.col[ORC_CPOLA] = col_pol_ang; k.col[ORC_CREFW] = col_ref_wavelength;
    k.col[ORC_CCURV] = col_sp_curvature; k.col[ORC_CLW] = col_line_width;
    k.col[ORC_CINC] = col_freq_inc;
    for (s = 0; s < num_sources; ++s)
    {
        const int* nv = num_valid + (size_t) s * ORC_SKY_NUM_TYPES;
        const int n_i = nv[ORC_SKY_I];
        const int n_ref = nv[ORC_SKY_REF_HZ], n_inc = nv[ORC_SKY_INC_HZ];
        const int n_pola = nv[ORC_SKY_POLA], n_polf = nv[ORC_SKY_POLF];
        REAL iquv[4] = {0, 0, 0, 0}, diff = (REAL) 1e38, f0 = 0;
        int j, chan = 0;
        /* nearest reference channel */
        for (j = 0; j < n_i; ++j)
        {
            const REAL tf = (n_inc == 1 && n_ref == 1) ?
                    ORC_T(sky_at)(&k, col_ref_freq, s) +
                    j * ORC_T(sky_at)(&k, col_freq_inc, s) :
                    ORC_T(sky_at)(&k, col_ref_freq + j, s);
            const REAL d = (REAL) fabs(tf - freq_hz);
            if (d < diff)
            {
                diff = d;
                chan = j;
                f0 = tf;
            }
        }
        for (j = 0; j < 4; ++j)
        {
            const int n = nv[ORC_SKY_I + j];
            if (n > 0)
                iquv[j] = ORC_T(sky_at)(&k, k.col[ORC_CI + j] +
                        (chan < n ? chan : 0), s);
            iquv[j] = ORC_T(nan0)(iquv[j]);
        }
        if (n_pola > 0 && n_polf > 0 && (nv[ORC_SKY_Q] <= 0 ||
                nv[ORC_SKY_U] <= 0))
        {
            const REAL ang = ORC_T(sky_at)(&k, col_pol_ang +
                    (chan < n_pola ? chan : 0), s);
            const REAL frac = ORC_T(sky_at)(&k, col_pol_frac +
                    (chan < n_polf ? chan : 0), s);
            const REAL sn = (REAL) sin(2 * ang), cs = (REAL) cos(2 * ang);
            iquv[1] = frac * iquv[0] * cs;
            iquv[2] = frac * iquv[0] * sn;
        }
        if (f0 == (REAL) 0)
        {
            out_i[s] = iquv[0]; out_q[s] = iquv[1];
            out_u[s] = iquv[2]; out_v[s] = iquv[3];
            continue;
        }
        {
            const REAL i_out = ORC_T(stokes_i_at)(&k, nv, s, iquv[0],
                    freq_hz, f0);
            const REAL scale = iquv[0] != (REAL) 0 ? i_out / iquv[0] : 0;
            if (nv[ORC_SKY_RM] > 0)
            {
                const REAL rm = ORC_T(nan0)(
                        ORC_T(sky_at)(&k, col_rot_meas, s));
                const REAL lambda = ((REAL) ORC_C0_M_PER_S) / freq_hz;
                REAL chi0, frac;
                if (n_pola <= 0 || n_polf <= 0)
                {
                    const REAL lambda0 = nv[ORC_SKY_REF_WAVE] > 0 ?
                            ORC_T(sky_at)(&k, col_ref_wavelength, s) :
                            ((REAL) ORC_C0_M_PER_S) / f0;
                    const REAL f_lambda0 = ((REAL) ORC_C0_M_PER_S) / lambda0;
                    const REAL i_ref = ORC_T(stokes_i_at)(&k, nv, s,
                            iquv[0], freq_hz, f_lambda0);
                    chi0 = (REAL) 0.5 * (REAL) atan2(iquv[2], iquv[1]) -
                            lambda0 * lambda0 * rm;
                    frac = (REAL) sqrt(iquv[1] * iquv[1] +
                            iquv[2] * iquv[2]) / i_ref;
                }
                else
                {
                    chi0 = ORC_T(sky_at)(&k, col_pol_ang +
                            (chan < n_pola ? chan : 0), s);
                    frac = ORC_T(sky_at)(&k, col_pol_frac +
                            (chan < n_polf ? chan : 0), s);
                }
                {
                    const REAL chi = chi0 + rm * (lambda * lambda);
                    out_q[s] = frac * i_out * (REAL) cos(2 * chi);
                    out_u[s] = frac * i_out * (REAL) sin(2 * chi);
                }
            }
            else
            {
                out_q[s] = scale * iquv[1];
                out_u[s] = scale * iquv[2];
            }
            out_i[s] = i_out;
            out_v[s] = scale * iquv[3];
        }
    }
}

/* Cable-length phase per station: J[p][s] <- diag(e^{i k dx_p},
 * e^{i k dy_p}) J[p][s] for a matrix Jones (an absent polarisation keeps
 * gain 1), J[p][s] <- e^{i k dx_p} J[p][s] for a scalar Jones (nothing
 * without x errors); k = 2 pi f / c
 * (interferometer/define_jones_apply_cable_length_errors.h:3-74). */
void ORC_FN(orc_cable_length_errors)(int matrix, int num_sources,
        int num_stations, REAL wavenumber, const REAL* errors_x,
        const REAL* errors_y, REAL* jones)
{
    int p, s;
    for (p = 0; p < num_stations; ++p)
    {
        ORC_T(cx) gx = {1, 0}, gy = {1, 0};
        if (errors_x)
        {
            const REAL ph = wavenumber * errors_x[p];
            gx.re = ORC_COS(ph);
            gx.im = ORC_SIN(ph);
        }
        if (errors_y)
        {
            const REAL ph = wavenumber * errors_y[p];
            gy.re = ORC_COS(ph);
            gy.im = ORC_SIN(ph);
        }
        if (!matrix && !errors_x) return;
        for (s = 0; s < num_sources; ++s)
        {
            REAL* e = jones + (size_t) (matrix ? 8 : 2) *
                    ((size_t) num_sources * p + s);
            int k;
            if (!matrix)
            {
                ORC_T(cx) v = {e[0], e[1]};
                v = ORC_T(cmul)(gx, v);
                e[0] = v.re; e[1] = v.im;
                continue;
            }
            /* rows a, b scale by gx; rows c, d by gy */
            for (k = 0; k < 4; ++k)
            {
                ORC_T(cx) v = {e[2 * k], e[2 * k + 1]};
                v = ORC_T(cmul)(k < 2 ? gx : gy, v);
                e[2 * k] = v.re; e[2 * k + 1] = v.im;
            }
        }
    }
}

/* J[p][s] <- G_p J[p][s]: 2x2 matrix product for matrix Jones, complex
 * product for scalar Jones
 * (interferometer/define_jones_apply_station_gains.h:3-45). */
void ORC_FN(orc_station_gains)(int matrix, int num_sources,
        int num_stations, const REAL* gains, REAL* jones)
{
    int p, s;
    for (p = 0; p < num_stations; ++p)
        for (s = 0; s < num_sources; ++s)
        {
            REAL* e = jones + (size_t) (matrix ? 8 : 2) *
                    ((size_t) num_sources * p + s);
            if (!matrix)
            {
                ORC_T(cx) g = {gains[2 * p], gains[2 * p + 1]};
                ORC_T(cx) v = {e[0], e[1]};
                v = ORC_T(cmul)(g, v);
                e[0] = v.re; e[1] = v.im;
            }
            else
            {
                const ORC_T(mat) G = ORC_T(load_mat)(gains + 8 * p);
                const ORC_T(mat) M = ORC_T(load_mat)(e);
                ORC_T(mat) out;
                out.a = ORC_T(cadd)(ORC_T(cmul)(G.a, M.a),
                        ORC_T(cmul)(G.b, M.c));
                out.b = ORC_T(cadd)(ORC_T(cmul)(G.a, M.b),
                        ORC_T(cmul)(G.b, M.d));
                out.c = ORC_T(cadd)(ORC_T(cmul)(G.c, M.a),
                        ORC_T(cmul)(G.d, M.c));
                out.d = ORC_T(cadd)(ORC_T(cmul)(G.c, M.b),
                        ORC_T(cmul)(G.d, M.d));
                e[0] = out.a.re; e[1] = out.a.im; e[2] = out.b.re;
                e[3] = out.b.im; e[4] = out.c.re; e[5] = out.c.im;
                e[6] = out.d.re; e[7] = out.d.im;
            }
        }
}

#ifndef ORC_PHILOX_
#define ORC_PHILOX_
/* Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC11, 2011), restated
 * from the paper: ten rounds; each round multiplies counter words 0 and 2
 * by 0xD2511F53 and 0xCD9E8D57 into 64-bit products and mixes the high
 * halves with the other words and the round key; the key is bumped by the
 * Weyl constants 0x9E3779B9 and 0xBB67AE85 before every round after the
 * first. The reference calls Random123's implementation (its
 * extern/Random123/philox.h) through math/private_random_generators.h:17-35
 * with key {seed, 0xCAFEF00D} and counter {index, c1, c2, c3}. */
static void orc_philox4x32_10(const uint32_t ctr[4], uint32_t seed,
        uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = seed, k1 = 0xCAFEF00Du;
    int r;
    for (r = 0; r < 10; ++r)
    {
        uint64_t p0, p1;
        if (r > 0)
        {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        p0 = (uint64_t) 0xD2511F53u * c0;
        p1 = (uint64_t) 0xCD9E8D57u * c2;
        c0 = (uint32_t) (p1 >> 32) ^ c1 ^ k0;
        c1 = (uint32_t) p1;
        c2 = (uint32_t) (p0 >> 32) ^ c3 ^ k1;
        c3 = (uint32_t) p0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
#endif

/* Box-Muller pair from two 32-bit integers as the reference's CPU path
 * forms it (math/private_random_helpers.h:42-107): angle pi x with
 * x = u0 2^-31 + 2^-32 (u0 taken as a non-negative integer, so x lies in
 * (0, 2)), radius sqrt(-2 log(u1 2^-32 + 2^-33)). */
static void ORC_T(box_muller)(uint32_t u0, uint32_t u1, REAL* f0, REAL* f1)
{
    const REAL f_angle = (REAL) 1 / ((REAL) 1 + (REAL) 0x7FFFFFFFuL);
    const REAL f_unit = (REAL) 1 / ((REAL) 1 + (REAL) 0xFFFFFFFFuL);
    const REAL x = ((REAL) (long) u0 * f_angle) + (REAL) 0.5 * f_angle;
    const REAL y = ((REAL) u1 * f_unit) + (REAL) 0.5 * f_unit;
    REAL t = (REAL) ORC_PI, r;
    t *= x;
    *f0 = ORC_SIN(t);
    *f1 = ORC_COS(t);
    r = ORC_SQRT((REAL) -2 * ORC_LOG(y));
    *f0 *= r;
    *f1 *= r;
}

/* n Gaussian values of standard deviation std, four per Philox call with
 * counter {i / 4, c1, c2, c3} (mem/src/oskar_mem_random_gaussian.c:14-130,
 * CPU path). */
void ORC_FN(orc_random_gaussian)(unsigned int n, REAL* data,
        unsigned int seed, unsigned int c1, unsigned int c2,
        unsigned int c3, REAL std)
{
    unsigned int q, k;
    for (q = 0; 4 * (size_t) q < n; ++q)
    {
        const uint32_t ctr[4] = {q, c1, c2, c3};
        uint32_t u[4];
        REAL t[4];
        orc_philox4x32_10(ctr, seed, u);
        ORC_T(box_muller)(u[0], u[1], &t[0], &t[1]);
        ORC_T(box_muller)(u[2], u[3], &t[2], &t[3]);
        for (k = 0; k < 4 && 4 * q + k < n; ++k) data[4 * q + k] = std * t[k];
    }
}

/* Time-variable element gain and phase errors: a Gaussian pair (g, h) per
 * element from counter {i / 2, time_index, station_id, 0x12345678}, then
 * (gain + gain_error g) e^{i (phase + phase_error h)}
 * (telescope/station/src/oskar_evaluate_element_weights_errors.c:19-110,
 * define_evaluate_element_weights_errors.h:3-16). */
void ORC_FN(orc_element_weights_errors)(int n, const REAL* gain,
        const REAL* gain_error, const REAL* phase, const REAL* phase_error,
        unsigned int seed, int time_index, int station_id, REAL* errors)
{
    int i;
    ORC_FN(orc_random_gaussian)(2 * (unsigned int) n, errors, seed,
            (unsigned int) time_index, (unsigned int) station_id,
            0x12345678u, (REAL) 1);
    for (i = 0; i < n; ++i)
    {
        REAL re = errors[2 * i], ph = errors[2 * i + 1];
        re *= gain_error[i];
        re += gain[i];
        ph *= phase_error[i];
        ph += phase[i];
        errors[2 * i] = ORC_COS(ph) * re;
        errors[2 * i + 1] = ORC_SIN(ph) * re;
    }
}

/* Beam-pattern auto power of one source's Jones terms: J B J^H, or |J|^2
 * for scalar Jones (correlate/define_evaluate_auto_power.h:3-40). */
void ORC_FN(orc_auto_power)(int matrix, int n, int offset_in,
        const REAL* jones, REAL I, REAL Q, REAL U, REAL V, int offset_out,
        REAL* out)
{
    int i;
    for (i = 0; i < n; ++i)
    {
        if (matrix)
        {
            const ORC_T(mat) J = ORC_T(load_mat)(jones + 8 *
                    (size_t) (i + offset_in));
            const ORC_T(mat) r = ORC_T(mul_herm)(
                    ORC_T(mul_brightness)(J, I, Q, U, V), J);
            REAL* o = out + 8 * (size_t) (i + offset_out);
            o[0] = r.a.re; o[1] = r.a.im; o[2] = r.b.re; o[3] = r.b.im;
            o[4] = r.c.re; o[5] = r.c.im; o[6] = r.d.re; o[7] = r.d.im;
        }
        else
        {
            const REAL* j = jones + 2 * (size_t) (i + offset_in);
            out[2 * (size_t) (i + offset_out)] = j[0] * j[0] + j[1] * j[1];
            out[2 * (size_t) (i + offset_out) + 1] = 0;
        }
    }
}

/* Beam-pattern cross power per source: norm sum_{p<q} (J_p B) J_q^H over
 * station pairs, or sum_{p<q} J_p conj(J_q) for scalar Jones, in the
 * reference's loop order (correlate/define_evaluate_cross_power.h:3-72;
 * norm = 2 / (N (N - 1)) from src/oskar_evaluate_cross_power.c:54). */
void ORC_FN(orc_cross_power)(int matrix, int num_sources, int num_stations,
        const REAL* jones, REAL I, REAL Q, REAL U, REAL V, REAL norm,
        int offset_out, REAL* out)
{
    int i, p, q;
    for (i = 0; i < num_sources; ++i)
    {
        if (matrix)
        {
            ORC_T(mat) sum;
            REAL* o = out + 8 * (size_t) (i + offset_out);
            sum.a.re = sum.a.im = sum.b.re = sum.b.im = 0;
            sum.c.re = sum.c.im = sum.d.re = sum.d.im = 0;
            for (p = 0; p < num_stations; ++p)
            {
                const ORC_T(mat) P = ORC_T(mul_brightness)(ORC_T(load_mat)(
                        jones + 8 * ((size_t) p * num_sources + i)),
                        I, Q, U, V);
                for (q = p + 1; q < num_stations; ++q)
                {
                    const ORC_T(mat) Qm = ORC_T(load_mat)(jones + 8 *
                            ((size_t) q * num_sources + i));
                    sum.a = ORC_T(cadd)(sum.a, ORC_T(cmulc)(P.a, Qm.a));
                    sum.a = ORC_T(cadd)(sum.a, ORC_T(cmulc)(P.b, Qm.b));
                    sum.b = ORC_T(cadd)(sum.b, ORC_T(cmulc)(P.a, Qm.c));
                    sum.b = ORC_T(cadd)(sum.b, ORC_T(cmulc)(P.b, Qm.d));
                    sum.c = ORC_T(cadd)(sum.c, ORC_T(cmulc)(P.c, Qm.a));
                    sum.c = ORC_T(cadd)(sum.c, ORC_T(cmulc)(P.d, Qm.b));
                    sum.d = ORC_T(cadd)(sum.d, ORC_T(cmulc)(P.c, Qm.c));
                    sum.d = ORC_T(cadd)(sum.d, ORC_T(cmulc)(P.d, Qm.d));
                }
            }
            o[0] = sum.a.re * norm; o[1] = sum.a.im * norm;
            o[2] = sum.b.re * norm; o[3] = sum.b.im * norm;
            o[4] = sum.c.re * norm; o[5] = sum.c.im * norm;
            o[6] = sum.d.re * norm; o[7] = sum.d.im * norm;
        }
        else
        {
            ORC_T(cx) sum = {0, 0};
            for (p = 0; p < num_stations; ++p)
            {
                ORC_T(cx) part = {0, 0};
                const REAL* jp = jones + 2 * ((size_t) p * num_sources + i);
                const ORC_T(cx) P = {jp[0], jp[1]};
                for (q = p + 1; q < num_stations; ++q)
                {
                    const REAL* jq = jones + 2 * ((size_t) q * num_sources + i);
                    const ORC_T(cx) Qc = {jq[0], jq[1]};
                    part = ORC_T(cadd)(part, ORC_T(cmulc)(P, Qc));
                }
                sum = ORC_T(cadd)(sum, part);
            }
            out[2 * (size_t) (i + offset_out)] = sum.re * norm;
            out[2 * (size_t) (i + offset_out) + 1] = sum.im * norm;
        }
    }
}
