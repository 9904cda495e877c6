/* TEST INFRASTRUCTURE ONLY — part of the parity oracle, never linked by the product.
 *
 * CPU restatement of the reference solver's numerical stages, written as a
 * macro template (define OR_REAL and OR_NS(name) before including, after
 * including fft_engine.h with the same real type).  With OR_REAL=float it
 * follows the reference's single-worker operation order exactly, so its
 * outputs can be compared bit-for-bit with the compiled reference core; with
 * OR_REAL=double it is the FP64 CPU oracle.
 *
 * Every stage cites the lines of updc/c_core/updc_core.c it restates.
 */

typedef struct {
    int W, H, iw, ih, nexp, FW, FH, transposed;
    size_t nout, nin, nf, nc;
    /* per exposure */
    OR_REAL *background, *pedestal, *mean_offset;
    int *psf_w, *psf_h;
    OR_REAL **spectrum;           /* nc complex (interleaved) */
    const uint32_t **offset;      /* nin+1, decoded LinkMap */
    const uint32_t **target;      /* nlinks, absolute */
    const float **frac;           /* nlinks */
    /* planes */
    OR_REAL *sci, *wht;           /* nexp*nin */
    uint8_t *frozen;              /* nexp*nin */
    OR_REAL *estimate, *coverage, *denominator, *correction, *blur, *scatter;
    OR_REAL *fft_image, *fft_freq, *estimate_freq, *partial;
    OR_REAL weight_scale, max_sensitivity;
    FE_NS(plan2d) *plan;
    /* per-iteration diagnostics of the last iteration */
    uint64_t *new_frozen, *total_frozen;
    OR_REAL *min_raw_mu;
    OR_REAL last_sum;
    uint64_t last_negative;
    char error[256];
} OR_NS(solver);

static int OR_NS(fail)(OR_NS(solver) *s, const char *msg) {
    snprintf(s->error, sizeof(s->error), "%s", msg);
    return -1;
}

/* core:777-789 Neumaier sum in the working precision */
static int OR_NS(psf_sum)(const float *psf, size_t count, OR_REAL *out) {
    OR_REAL sum = 0, comp = 0;
    for (size_t p = 0; p < count; ++p) {
        const OR_REAL v = (OR_REAL)psf[p];
        if (!isfinite(v) || v < 0) return -1;
        const OR_REAL t = sum + v;
        if (fabs((double)sum) >= fabs((double)v)) comp += (sum - t) + v;
        else comp += (v - t) + sum;
        sum = t;
    }
    *out = sum + comp;
    return 0;
}

/* core:807-822 normalise, centre-wrap (optionally transposed) and R2C */
static int OR_NS(prepare_psf)(OR_NS(solver) *s, int k, const float *psf) {
    const int pw = s->psf_w[k], ph = s->psf_h[k];
    OR_REAL sum;
    if (OR_NS(psf_sum)(psf, (size_t)pw * ph, &sum)) return OR_NS(fail)(s, "invalid PSF pixel");
    if (!(sum > 0) || !isfinite(sum)) return OR_NS(fail)(s, "PSF sum is zero/non-finite");
    const OR_REAL inv = (OR_REAL)1 / sum;
    memset(s->fft_image, 0, s->nf * sizeof(OR_REAL));
    const int fwid = s->transposed ? ph : pw, fhei = s->transposed ? pw : ph;
    for (int y = 0; y < fhei; ++y)
        for (int x = 0; x < fwid; ++x) {
            const int yy = (y - fhei / 2 + s->FH) % s->FH;
            const int xx = (x - fwid / 2 + s->FW) % s->FW;
            const size_t src = s->transposed ? (size_t)x * pw + y : (size_t)y * pw + x;
            s->fft_image[(size_t)yy * s->FW + xx] = (OR_REAL)psf[src] * inv;
        }
    FE_NS(exec_r2c)(s->plan, s->fft_image, s->spectrum[k]);
    return 0;
}

/* core:728-737 / 748-751 zero-pad the W x H plane into FW x FH and R2C */
static void OR_NS(forward_target)(OR_NS(solver) *s, const OR_REAL *src, OR_REAL *dest) {
    memset(s->fft_image, 0, s->nf * sizeof(OR_REAL));
    for (int y = 0; y < s->H; ++y)
        memcpy(s->fft_image + (size_t)y * s->FW, src + (size_t)y * s->W, (size_t)s->W * sizeof(OR_REAL));
    FE_NS(exec_r2c)(s->plan, s->fft_image, dest);
}

/* core:738-744 / 761-767 C2R of fft_freq, crop to W x H, multiply by 1/nf */
static void OR_NS(inverse_crop)(OR_NS(solver) *s, OR_REAL *dest) {
    FE_NS(exec_c2r)(s->plan, s->fft_freq, s->fft_image);
    const OR_REAL scale = (OR_REAL)1 / (OR_REAL)s->nf;
    for (int y = 0; y < s->H; ++y)
        for (int x = 0; x < s->W; ++x)
            dest[(size_t)y * s->W + x] = s->fft_image[(size_t)y * s->FW + x] * scale;
}

/* core:988-995 dest += conj(kernel) * src, products (ac+bd, bc-ad) */
static void OR_NS(accumulate_adjoint)(OR_NS(solver) *s, OR_REAL *dest, const OR_REAL *src, const OR_REAL *kernel) {
    for (size_t p = 0; p < s->nc; ++p) {
        const OR_REAL a = src[2 * p], b = src[2 * p + 1], c = kernel[2 * p], d = kernel[2 * p + 1];
        dest[2 * p] += a * c + b * d;
        dest[2 * p + 1] += b * c - a * d;
    }
}

/* core:378-424 weight scale = median of every 64th positive WHT; mask; W /= scale */
static int OR_NS(weight_scale)(OR_NS(solver) *s) {
    size_t cap = (size_t)s->nexp * (s->nin / 64 + 1), n = 0;
    float *sample = (float *)malloc(cap * sizeof(float));
    for (int k = 0; k < s->nexp; ++k) {
        const OR_REAL *w = s->wht + (size_t)k * s->nin;
        for (size_t p = 0; p < s->nin; p += 64)
            if (isfinite(w[p]) && w[p] > 0) sample[n++] = (float)w[p];
    }
    if (!n) { free(sample); return OR_NS(fail)(s, "all input WHT pixels are zero"); }
    qsort(sample, n, sizeof(float), orc_cmp_float);
    s->weight_scale = (OR_REAL)sample[n / 2];
    free(sample);
    if (!(s->weight_scale > 0) || !isfinite(s->weight_scale)) return OR_NS(fail)(s, "invalid WHT normalization");
    for (int k = 0; k < s->nexp; ++k) {
        OR_REAL *in = s->sci + (size_t)k * s->nin, *w = s->wht + (size_t)k * s->nin;
        for (size_t p = 0; p < s->nin; ++p) {
            if (!isfinite(in[p]) || !isfinite(w[p]) || !(w[p] > 0)) { in[p] = 0; w[p] = 0; continue; }
            w[p] /= s->weight_scale;
            if (!isfinite(w[p]) || !(w[p] > 0)) return OR_NS(fail)(s, "invalid normalized WHT");
            const OR_REAL y = in[p] + s->pedestal[k];
            if (!isfinite(y) || y < 0) return OR_NS(fail)(s, "negative/non-finite y_eff reached solver");
        }
    }
    return 0;
}

/* core:947-973 initial signed drizzle estimate and coverage (serial order) */
static int OR_NS(drizzle)(OR_NS(solver) *s) {
    OR_REAL *data = (OR_REAL *)calloc(s->nout, sizeof(OR_REAL));
    OR_REAL *bkg = (OR_REAL *)calloc(s->nout, sizeof(OR_REAL));
    memset(s->coverage, 0, s->nout * sizeof(OR_REAL));
    for (int k = 0; k < s->nexp; ++k) {
        const OR_REAL *in = s->sci + (size_t)k * s->nin, *w = s->wht + (size_t)k * s->nin;
        const uint32_t *off = s->offset[k], *tg = s->target[k];
        const float *fr = s->frac[k];
        for (size_t p = 0; p < s->nin; ++p) {
            if (!(w[p] > 0) || off[p] == off[p + 1]) continue;
            const OR_REAL wp = w[p];
            for (uint32_t z = off[p]; z < off[p + 1]; ++z) {
                const uint32_t t = tg[z];
                const OR_REAL q = (OR_REAL)fr[z] * wp;
                s->coverage[t] += q;
                data[t] = OR_FMA(q, in[p], data[t]);
                bkg[t] = OR_FMA(q, s->background[k], bkg[t]);
            }
        }
    }
    for (size_t t = 0; t < s->nout; ++t) {
        if (s->coverage[t] > (OR_REAL)1e-12f) {
            s->estimate[t] = data[t] / s->coverage[t] - bkg[t] / s->coverage[t];
            if (!isfinite(s->estimate[t])) { free(data); free(bkg); return OR_NS(fail)(s, "non-finite signed initial estimate"); }
        } else s->estimate[t] = 0;
    }
    free(data); free(bkg);
    return 0;
}

/* core:1052-1082 D = crop(C2R(sum_k conj(K_k) R2C(pad(S_k^T W_k))))/nf */
static int OR_NS(denominator_stage)(OR_NS(solver) *s) {
    memset(s->partial, 0, 2 * s->nc * sizeof(OR_REAL));
    for (int k = 0; k < s->nexp; ++k) {
        const OR_REAL *w = s->wht + (size_t)k * s->nin;
        const uint32_t *off = s->offset[k], *tg = s->target[k];
        const float *fr = s->frac[k];
        memset(s->scatter, 0, s->nout * sizeof(OR_REAL));
        for (size_t p = 0; p < s->nin; ++p) {
            if (!(w[p] > 0) || off[p] == off[p + 1]) continue;
            const OR_REAL wp = w[p];
            for (uint32_t z = off[p]; z < off[p + 1]; ++z)
                s->scatter[tg[z]] = OR_FMA((OR_REAL)fr[z], wp, s->scatter[tg[z]]);
        }
        OR_NS(forward_target)(s, s->scatter, s->fft_freq);
        OR_NS(accumulate_adjoint)(s, s->partial, s->fft_freq, s->spectrum[k]);
    }
    for (size_t p = 0; p < 2 * s->nc; ++p) s->fft_freq[p] = (OR_REAL)0 + s->partial[p];
    OR_NS(inverse_crop)(s, s->denominator);
    s->max_sensitivity = 0;
    for (size_t t = 0; t < s->nout; ++t) if (s->denominator[t] > s->max_sensitivity) s->max_sensitivity = s->denominator[t];
    if (!(s->max_sensitivity > 0) || !isfinite(s->max_sensitivity)) return OR_NS(fail)(s, "invalid H^T W sensitivity");
    return 0;
}

/* H^T v = crop(C2R(sum_k conj(K_k) R2C(pad(S_k^T v_k))))/nf for detector
 * planes v (nexp x nin): the scatter of core:1175-1176 (fmaf in link order),
 * the adjoint accumulation of core:988-995 and the reduction of
 * core:1280-1287, applied to arbitrary detector values (the differentiable
 * model's residual W(ratio - 1)).  Result in dest (nout). */
static void OR_NS(adjoint)(OR_NS(solver) *s, const OR_REAL *v_all, OR_REAL *dest) {
    memset(s->partial, 0, 2 * s->nc * sizeof(OR_REAL));
    for (int k = 0; k < s->nexp; ++k) {
        const OR_REAL *v = v_all + (size_t)k * s->nin;
        const uint32_t *off = s->offset[k], *tg = s->target[k];
        const float *fr = s->frac[k];
        memset(s->scatter, 0, s->nout * sizeof(OR_REAL));
        for (size_t p = 0; p < s->nin; ++p) {
            if (off[p] == off[p + 1]) continue;
            const OR_REAL vp = v[p];
            for (uint32_t z = off[p]; z < off[p + 1]; ++z)
                s->scatter[tg[z]] = OR_FMA((OR_REAL)fr[z], vp, s->scatter[tg[z]]);
        }
        OR_NS(forward_target)(s, s->scatter, s->fft_freq);
        OR_NS(accumulate_adjoint)(s, s->partial, s->fft_freq, s->spectrum[k]);
    }
    for (size_t p = 0; p < 2 * s->nc; ++p) s->fft_freq[p] = (OR_REAL)0 + s->partial[p];
    OR_NS(inverse_crop)(s, dest);
}

/* core:1152-1177 fused detector loop of one exposure given its blur plane.
 * Writes scatter (zeroed first) and updates the freeze mask. */
static int OR_NS(detector)(const OR_NS(solver) *s, int k, const OR_REAL *blur, OR_REAL *scatter,
                           uint64_t *nnew_out, uint64_t *ntotal_out, OR_REAL *min_out, char *err, size_t errcap) {
    const OR_REAL *in = s->sci + (size_t)k * s->nin, *w = s->wht + (size_t)k * s->nin;
    uint8_t *frozen = s->frozen + (size_t)k * s->nin;
    const uint32_t *off = s->offset[k], *tg = s->target[k];
    const float *fr = s->frac[k];
    memset(scatter, 0, s->nout * sizeof(OR_REAL));
    uint64_t nnew = 0, ntotal = 0;
    OR_REAL min_raw_mu = (OR_REAL)INFINITY;
    for (size_t p = 0; p < s->nin; ++p) {
        if (!(w[p] > 0) || off[p] == off[p + 1]) continue;
        OR_REAL pred = 0;
        for (uint32_t z = off[p]; z < off[p + 1]; ++z) pred = OR_FMA((OR_REAL)fr[z], blur[tg[z]], pred);
        const OR_REAL raw_mu = pred + s->mean_offset[k];
        if (!isfinite(raw_mu)) { snprintf(err, errcap, "non-finite forward mean"); return -1; }
        if (raw_mu < min_raw_mu) min_raw_mu = raw_mu;
        if (!frozen[p] && !(raw_mu > 0)) { frozen[p] = 1; ++nnew; }
        OR_REAL ratio;
        if (frozen[p]) { ++ntotal; ratio = 1; }
        else {
            const OR_REAL y = in[p] + s->pedestal[k];
            ratio = y / raw_mu;
            if (!isfinite(ratio)) { snprintf(err, errcap, "non-finite y/raw_mu ratio"); return -1; }
        }
        const OR_REAL wr = w[p] * ratio;
        for (uint32_t z = off[p]; z < off[p + 1]; ++z) scatter[tg[z]] = OR_FMA((OR_REAL)fr[z], wr, scatter[tg[z]]);
    }
    *nnew_out = nnew; *ntotal_out = ntotal; *min_out = min_raw_mu;
    return 0;
}

/* core:1437-1456 multiplicative update */
static int OR_NS(update)(OR_NS(solver) *s) {
    OR_REAL sum = 0;
    uint64_t nneg = 0;
    for (size_t t = 0; t < s->nout; ++t) {
        if (s->denominator[t] > (OR_REAL)1e-8f) {
            OR_REAL factor = s->correction[t] / s->denominator[t];
            if (!isfinite(factor)) return OR_NS(fail)(s, "non-finite multiplicative correction");
            if (factor < 0) {
                if (s->correction[t] < (OR_REAL)-1.0e-6f * s->max_sensitivity)
                    return OR_NS(fail)(s, "substantially negative multiplicative correction");
                factor = 0;
            }
            s->estimate[t] *= factor;
        } else s->estimate[t] = 0;
        if (!isfinite(s->estimate[t])) return OR_NS(fail)(s, "non-finite signed UPDC estimate");
        sum += s->estimate[t];
        if (s->estimate[t] < 0) nneg++;
    }
    s->last_sum = sum;
    s->last_negative = nneg;
    return 0;
}

/* core:1410-1456 one iteration */
static int OR_NS(iterate)(OR_NS(solver) *s) {
    OR_NS(forward_target)(s, s->estimate, s->estimate_freq);
    memset(s->partial, 0, 2 * s->nc * sizeof(OR_REAL));
    for (int k = 0; k < s->nexp; ++k) {
        /* core:753-760 forward product (ac-bd, ad+bc), then C2R + crop */
        const OR_REAL *sp = s->spectrum[k];
        for (size_t p = 0; p < s->nc; ++p) {
            const OR_REAL a = s->estimate_freq[2 * p], b = s->estimate_freq[2 * p + 1];
            const OR_REAL c = sp[2 * p], d = sp[2 * p + 1];
            s->fft_freq[2 * p] = a * c - b * d;
            s->fft_freq[2 * p + 1] = a * d + b * c;
        }
        OR_NS(inverse_crop)(s, s->blur);
        if (OR_NS(detector)(s, k, s->blur, s->scatter, &s->new_frozen[k], &s->total_frozen[k],
                            &s->min_raw_mu[k], s->error, sizeof(s->error))) return -1;
        OR_NS(forward_target)(s, s->scatter, s->fft_freq);
        OR_NS(accumulate_adjoint)(s, s->partial, s->fft_freq, sp);
    }
    for (size_t p = 0; p < 2 * s->nc; ++p) s->fft_freq[p] = (OR_REAL)0 + s->partial[p];
    OR_NS(inverse_crop)(s, s->correction);
    return OR_NS(update)(s);
}
