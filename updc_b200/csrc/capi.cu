// C ABI of the B200 engine (include/updc_b200.h) and the UPDC_ALL driver.
#include <sys/resource.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/updc_b200.h"
#include "engine.cuh"
#include "linkmap.cuh"
#include "preprocess.cuh"

using namespace updc;

struct updc_engine {
    std::unique_ptr<Engine> owned;  // null for the field handles of a batch
    Engine *e = nullptr;
    EngineOptions opt;
    int nexp = 0;
};

struct updc_batch {
    std::unique_ptr<Batch> b;
    std::vector<std::unique_ptr<updc_engine>> views;
};

namespace {

thread_local std::string g_last_error;

int fail_status(const std::exception &ex) {
    g_last_error = ex.what();
    const Error *e = dynamic_cast<const Error *>(&ex);
    return e && e->code ? e->code : 1;
}

template <class F> int guarded(F &&f) {
    try {
        g_last_error.clear();
        f();
        return 0;
    } catch (const std::exception &ex) {
        return fail_status(ex);
    } catch (...) {
        g_last_error = "unknown failure";
        return 1;
    }
}

EngineOptions to_options(const updc_options *o) {
    EngineOptions r;
    if (!o) return r;
    r.form = o->form;
    r.compensated_mu = o->compensated_mu;
    r.use_graph = o->use_graph;
    r.device = o->device;
    r.reuse_links = o->reuse_links;
    r.verbose = o->verbose;
    r.fft_width = o->fft_width;
    r.fft_height = o->fft_height;
    r.stage_timing = o->stage_timing;
    r.autotune = o->autotune;
    r.retune = o->retune;
    r.tune_cache_dir = o->tune_cache_dir ? o->tune_cache_dir : "";
    r.fft_linear = o->fft_linear;
    return r;
}

double wall() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}  // namespace

extern "C" {

const char *updc_version(void) { return "updc_b200 1.0 (sm_100a)"; }
const char *updc_last_error(void) { return g_last_error.c_str(); }

void updc_default_options(updc_options *o) {
    if (!o) return;
    EngineOptions d;
    o->form = d.form;
    o->compensated_mu = d.compensated_mu;
    o->use_graph = d.use_graph;
    o->device = d.device;
    o->reuse_links = d.reuse_links;
    o->verbose = d.verbose;
    o->fft_width = d.fft_width;
    o->fft_height = d.fft_height;
    o->stage_timing = d.stage_timing;
    o->autotune = d.autotune;
    o->retune = d.retune;
    o->tune_cache_dir = nullptr;
    o->fft_linear = d.fft_linear;
}

int updc_create(const updc_options *opt, updc_engine **out) {
    return guarded([&] {
        if (!out) throw Error(1, "null output handle");
        *out = nullptr;
        EngineOptions o = to_options(opt);
        if (o.form < 0 || o.form > 3) throw Error(1, "unknown precision form");
        updc_engine *h = new updc_engine;
        h->opt = o;
        try {
            h->owned = make_engine(o);
            h->e = h->owned.get();
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int updc_destroy(updc_engine *h) {
    return guarded([&] {
        if (h && !h->owned) throw Error(1, "a batch field handle is owned by its batch");
        delete h;
    });
}

int updc_load_manifest(updc_engine *h, const char *manifest, int W, int H, int iw, int ih, int nexp, int tr) {
    return guarded([&] {
        if (!h || !manifest) throw Error(1, "null argument");
        h->e->load(manifest, W, H, iw, ih, nexp, tr);
        h->nexp = nexp;
    });
}

int updc_setup(updc_engine *h) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->setup();
    });
}

int updc_iterate(updc_engine *h, int n, int check_each, updc_iter_stats *stats, uint64_t *new_frozen,
                 uint64_t *total_frozen, double *min_raw_mu) {
    return guarded([&] {
        if (!h || n < 0) throw Error(1, "invalid arguments");
        std::vector<IterationRecord> rec;
        h->e->iterate(n, check_each != 0, &rec);
        for (int i = 0; i < n && i < (int)rec.size(); ++i) {
            if (stats) {
                stats[i].seconds = rec[i].seconds;
                stats[i].signed_sum = rec[i].signed_sum;
                stats[i].negative = rec[i].negative;
                for (int s = 0; s < 8; ++s) stats[i].stage_seconds[s] = rec[i].stage_seconds[s];
            }
            for (int k = 0; k < h->nexp; ++k) {
                if (new_frozen) new_frozen[(size_t)i * h->nexp + k] = rec[i].new_frozen[k];
                if (total_frozen) total_frozen[(size_t)i * h->nexp + k] = rec[i].total_frozen[k];
                if (min_raw_mu) min_raw_mu[(size_t)i * h->nexp + k] = rec[i].min_raw_mu[k];
            }
        }
    });
}

int updc_read_plane(updc_engine *h, int which, int k, void *host, int as_double) {
    return guarded([&] {
        if (!h || !host) throw Error(1, "null argument");
        h->e->read_plane(which, k, host, as_double);
    });
}
int updc_write_plane(updc_engine *h, int which, int k, const void *host, int as_double) {
    return guarded([&] {
        if (!h || !host) throw Error(1, "null argument");
        h->e->write_plane(which, k, host, as_double);
    });
}
double updc_scalar(updc_engine *h, int which) { return h ? h->e->scalar(which) : 0.0; }
int updc_fft_radices(updc_engine *h, int axis, int *radices, int capacity, int *count) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        const FftChoice &c = h->e->fft_choice();
        const std::vector<int> &r = axis == 0 ? c.row_radices : c.col_radices;
        for (int i = 0; i < (int)r.size() && i < capacity; ++i) radices[i] = r[i];
        if (count) *count = (int)r.size();
    });
}
size_t updc_device_bytes(updc_engine *h) { return h ? h->e->device_bytes() : 0; }
int updc_set_stage_timing(updc_engine *h, int on) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->set_stage_timing(on);
    });
}

int updc_stage_forward(updc_engine *h) {
    return guarded([&] { h->e->stage_forward(0); });
}
int updc_stage_detector(updc_engine *h, uint64_t *nn, uint64_t *nt, double *mn) {
    return guarded([&] {
        IterationRecord r;
        h->e->stage_detector(0, &r);
        for (int k = 0; k < h->nexp; ++k) {
            if (nn) nn[k] = r.new_frozen[k];
            if (nt) nt[k] = r.total_frozen[k];
            if (mn) mn[k] = r.min_raw_mu[k];
        }
    });
}
int updc_stage_correction(updc_engine *h) {
    return guarded([&] { h->e->stage_correction(); });
}
int updc_stage_update(updc_engine *h, double *sum, uint64_t *neg) {
    return guarded([&] {
        IterationRecord r;
        h->e->stage_update(&r);
        if (sum) *sum = r.signed_sum;
        if (neg) *neg = r.negative;
    });
}

int updc_set_exposure_offsets(updc_engine *h, int k, double background, double pedestal) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->set_exposure_offsets(k, background, pedestal);
    });
}
int updc_set_psf(updc_engine *h, int k, const void *psf, int pw, int ph, int as_double) {
    return guarded([&] {
        if (!h || !psf) throw Error(1, "null handle or PSF");
        h->e->set_psf(k, psf, pw, ph, as_double);
    });
}
int updc_nll(updc_engine *h, double *terms) {
    return guarded([&] {
        if (!h || !terms) throw Error(1, "null handle or output");
        h->e->nll(terms);
    });
}
int updc_nll_partials(updc_engine *h, double *out, size_t capacity, size_t *count) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        const std::vector<double> &p = h->e->nll_partials();
        if (out) memcpy(out, p.data(), std::min(capacity, p.size()) * sizeof(double));
        if (count) *count = p.size();
    });
}
int updc_nll_adjoint(updc_engine *h) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->nll_adjoint();
    });
}
int updc_psf_gradient(updc_engine *h, int k, double *out) {
    return guarded([&] {
        if (!h || !out) throw Error(1, "null handle or output");
        h->e->psf_gradient(k, out);
    });
}
int updc_copy_plane_device(updc_engine *h, int which, int k, void *dptr, int to_engine, int as_double, void *stream) {
    return guarded([&] {
        if (!h || !dptr) throw Error(1, "null handle or device pointer");
        h->e->copy_plane_device(which, k, dptr, to_engine, as_double, static_cast<cudaStream_t>(stream));
    });
}

int updc_set_active_exposures(updc_engine *h, int first, int count) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->set_active_exposures(first, count);
    });
}
int updc_refresh_sensitivity(updc_engine *h) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->refresh_sensitivity();
    });
}
int updc_finish_shard_setup(updc_engine *h) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->finish_shard_setup();
    });
}
int updc_plane_device_pointer(updc_engine *h, int which, void **device_ptr) {
    return guarded([&] {
        if (!h || !device_ptr) throw Error(1, "null handle or output pointer");
        *device_ptr = h->e->plane_device(which);
    });
}
int updc_engine_stream(updc_engine *h, void **stream) {
    return guarded([&] {
        if (!h || !stream) throw Error(1, "null handle or output pointer");
        *stream = static_cast<void *>(h->e->stream());
    });
}
int updc_enqueue_partial(updc_engine *h) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->enqueue_partial();
    });
}
int updc_enqueue_update(updc_engine *h) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        h->e->enqueue_update();
    });
}
int updc_finish_iteration(updc_engine *h, double *sum, uint64_t *neg, uint64_t *nn, uint64_t *nt, double *mn) {
    return guarded([&] {
        if (!h) throw Error(1, "null handle");
        IterationRecord r;
        h->e->finish_iteration(&r);
        if (sum) *sum = r.signed_sum;
        if (neg) *neg = r.negative;
        for (int k = 0; k < h->nexp; ++k) {
            if (nn) nn[k] = r.new_frozen[k];
            if (nt) nt[k] = r.total_frozen[k];
            if (mn) mn[k] = r.min_raw_mu[k];
        }
    });
}

int updc_save_state(updc_engine *h, const char *path, uint64_t iteration) {
    return guarded([&] {
        if (!h || !path) throw Error(1, "null argument");
        h->e->save_state(path, iteration);
    });
}
int updc_load_state(updc_engine *h, const char *path, uint64_t *iteration) {
    return guarded([&] {
        if (!h || !path) throw Error(1, "null argument");
        h->e->load_state(path, iteration);
    });
}

uint64_t updc_link_count(updc_engine *h, int k) { return h ? h->e->link_count(k) : 0; }
int updc_link_encoding(updc_engine *h, int k) { return h ? h->e->link_encoding(k) : 0; }
int updc_decode_links(updc_engine *h, int k, uint32_t *targets) {
    return guarded([&] { h->e->decode_links(k, targets); });
}

int updc_update_noalloc(const float *correction, const float *denominator, float *estimate, uint64_t n,
                        float max_sensitivity, void *stream, double *signed_sum, uint64_t *negative) {
    return guarded([&] {
        update_noalloc(correction, denominator, estimate, n, max_sensitivity, static_cast<cudaStream_t>(stream),
                       signed_sum, negative);
    });
}

int updc_build_linkmap(const char *vertices, const char *links, int iw, int ih, int W, int H, uint64_t *nlinks,
                       int *encoding) {
    return guarded([&] {
        cudaStream_t s;
        UPDC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        LinkBuildStats st;
        try {
            linkmap_build(vertices, links, iw, ih, W, H, s, &st);
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
        if (nlinks) *nlinks = st.nlinks;
        if (encoding) *encoding = (int)st.encoding;
    });
}

int updc_preprocess_exposure(const float *science, const uint32_t *dq, const double *var_poisson,
                             const double *var_rnoise, const double *var_flat, int64_t npix, int weight_mode,
                             uint32_t bad_dq_mask, double pedestal_sigma, const char *source, float *wht,
                             uint8_t *sky_mask, updc_preprocess_metrics *metrics, int device_pointers, void *stream) {
    return guarded([&] {
        if (npix <= 0) throw Error(1, "invalid exposure size");
        preprocess_exposure(science, dq, var_poisson, var_rnoise, var_flat, (size_t)npix, weight_mode, bad_dq_mask,
                            pedestal_sigma, source ? source : "", wht, sky_mask, metrics, device_pointers != 0,
                            (cudaStream_t)stream);
    });
}

int updc_robust_background(const float *science, const uint8_t *base_valid, int64_t npix, int max_iter,
                           uint8_t *mask, double *background, double *sigma, int *passes, int device_pointers,
                           void *stream) {
    return guarded([&] {
        if (npix <= 0) throw Error(1, "invalid exposure size");
        robust_background(science, base_valid, (size_t)npix, max_iter, mask, background, sigma, passes,
                          device_pointers != 0, (cudaStream_t)stream);
    });
}

float updc_polygon_area(const double *xy, int count) { return geometry_polygon_area_host(xy, count); }
float updc_overlap_area(const double *quad8, int x, int y) { return geometry_overlap_area_host(quad8, x, y); }
int updc_self_test(char *msg, size_t cap) {
    char local[256] = {0};
    const int rc = geometry_self_test(local, sizeof(local));
    if (msg && cap) snprintf(msg, cap, "%s", rc ? local : "UPDC B200 core self-test: OK");
    return rc;
}

int updc_device_wait_check(uint32_t polls) {
    return guarded([&] { device_wait_check(polls); });
}

// ---------------------------------------------------------------------------- batched fields
int updc_batch_create(const updc_options *opt, updc_batch **out) {
    return guarded([&] {
        if (!out) throw Error(1, "null output handle");
        *out = nullptr;
        EngineOptions o = to_options(opt);
        if (o.form < 0 || o.form > 3) throw Error(1, "unknown precision form");
        std::unique_ptr<updc_batch> b(new updc_batch);
        b->b = make_batch(o);
        *out = b.release();
    });
}
int updc_batch_destroy(updc_batch *b) {
    return guarded([&] { delete b; });
}
int updc_batch_add_field(updc_batch *b, const char *manifest, int W, int H, int iw, int ih, int nexp, int tr) {
    return guarded([&] {
        if (!b || !manifest) throw Error(1, "null argument");
        b->b->add_field(manifest, W, H, iw, ih, nexp, tr);
        std::unique_ptr<updc_engine> v(new updc_engine);
        v->e = &b->b->field(b->b->fields() - 1);
        v->nexp = nexp;
        b->views.push_back(std::move(v));
    });
}
int updc_batch_setup(updc_batch *b) {
    return guarded([&] {
        if (!b) throw Error(1, "null handle");
        b->b->setup();
    });
}
int updc_batch_fields(updc_batch *b) { return b ? b->b->fields() : 0; }
updc_engine *updc_batch_field(updc_batch *b, int i) {
    if (!b || i < 0 || i >= (int)b->views.size()) return nullptr;
    return b->views[i].get();
}
size_t updc_batch_units(updc_batch *b, int stage) { return b ? b->b->units(stage) : 0; }
int updc_batch_iterate(updc_batch *b, int n, int check_each, double *seconds, double *signed_sum, uint64_t *negative,
                       uint64_t *total_frozen) {
    return guarded([&] {
        if (!b) throw Error(1, "null handle");
        std::vector<BatchRecord> recs;
        b->b->iterate(n, check_each != 0, &recs);
        const int nf = b->b->fields();
        for (int i = 0; i < (int)recs.size(); ++i) {
            if (seconds) seconds[i] = recs[i].seconds;
            for (int f = 0; f < nf; ++f) {
                if (signed_sum) signed_sum[(size_t)i * nf + f] = recs[i].signed_sum[f];
                if (negative) negative[(size_t)i * nf + f] = recs[i].negative[f];
            }
            if (total_frozen) {
                const size_t ne = recs[i].total_frozen.size();
                for (size_t k = 0; k < ne; ++k) total_frozen[(size_t)i * ne + k] = recs[i].total_frozen[k];
            }
        }
    });
}

// ---------------------------------------------------------------------------- UPDC_ALL
int updc_all(const char *manifest, int width, int height, int input_width, int input_height, int exposures,
             int transpose_psf, int iterations, const char *iter_prefix, const char *weight_output,
             int fft_worker_count, int exposure_worker_count, int preprocess_worker_count, int plan_measure,
             int autotune, int retune_fft, const char *wisdom_path, int save_every) {
    return guarded([&] {
        (void)plan_measure;  // FFTW planner rigour: no counterpart (plans are timed by the autotuner)
        (void)wisdom_path;   // FFTW wisdom file: the autotuner keeps its own cache file instead
        if (width < 1 || height < 1 || input_width < 1 || input_height < 1 || exposures < 1 || iterations < 1 ||
            fft_worker_count < 1 || exposure_worker_count < 1 || preprocess_worker_count < 1 || save_every < 0)
            throw Error(1, "invalid dimensions/exposures/iterations/workers/save_every");
        const double total_start = wall();
        const char *pc = getenv("UPDC_PERSIST_CACHE");
        const bool persist = pc && strcmp(pc, "0") != 0;
        printf("Persistent C preprocessing cache: %s\n", persist ? "enabled" : "disabled");
        EngineOptions o;
        const char *form = getenv("UPDC_B200_FORM");
        if (form) o.form = atoi(form);
        o.reuse_links = persist ? 1 : 0;  // the reference rebuilds LinkMaps unless the cache is enabled
        o.verbose = 1;
        // FFT autotune with the reference's flags and cache root (updc_core.c:130-138, 242-291)
        o.autotune = autotune ? 1 : 0;
        o.retune = retune_fft ? 1 : 0;
        if (persist) {
            const char *slash = strrchr(manifest, '/');
            o.tune_cache_dir = slash ? std::string(manifest, slash - manifest) : std::string(".");
        }
        std::unique_ptr<Engine> e = make_engine(o);
        e->load(manifest, width, height, input_width, input_height, exposures, transpose_psf);
        const double setup_start = wall();
        e->setup();
        const double setup_time = wall() - setup_start;
        const int FW = (int)e->scalar(2), FH = (int)e->scalar(3);
        if (autotune)
            printf("FFT autotune %s %dx%d (%d plans timed, modelled %.3f ms/iteration)\n",
                   e->scalar(9) ? "persistent-cache hit:" : "selected", FW, FH, (int)e->scalar(8), e->scalar(10));
        printf("Background-aware UPDC (B200): %d exposures, input %dx%d, target %dx%d, FFT %dx%d, iterations %d\n",
               exposures, input_width, input_height, width, height, FW, FH, iterations);
        printf("WHT median normalization %.9g (%llu masked)\n", e->scalar(0), (unsigned long long)e->scalar(4));
        fflush(stdout);
        const std::string prefix = iter_prefix;
        FILE *freeze = fopen((prefix + "_mufreeze.csv").c_str(), "w");
        if (!freeze) throw Error(1, "cannot write freeze CSV");
        fprintf(freeze, "iteration,exposure,n_new_frozen,n_total_frozen,min_raw_mu,mu_marker,frozen_ratio\n");
        const size_t nout = (size_t)width * height;
        std::vector<float> plane(nout);
        std::vector<IterationRecord> recs;
        std::vector<double> iter_total(iterations), iter_output(iterations);
        for (int it = 1; it <= iterations; ++it) {
            const double t0 = wall();
            std::vector<IterationRecord> r;
            try {
                e->iterate(1, true, &r);
            } catch (...) {
                fclose(freeze);
                throw;
            }
            uint64_t nn = 0, nt = 0;
            double mn = INFINITY;
            for (int k = 0; k < exposures; ++k) {
                nn += r[0].new_frozen[k];
                nt += r[0].total_frozen[k];
                mn = std::min(mn, r[0].min_raw_mu[k]);
                fprintf(freeze, "%d,%d,%llu,%llu,%.9g,%.9g,1\n", it, k + 1, (unsigned long long)r[0].new_frozen[k],
                        (unsigned long long)r[0].total_frozen[k], (double)(float)r[0].min_raw_mu[k], (double)1.0e-12f);
            }
            const double t1 = wall();
            const bool save = it == iterations || (save_every > 0 && it % save_every == 0);
            if (save) {
                char path[4096];
                if (snprintf(path, sizeof(path), "%s_%02d.bin", iter_prefix, it) >= (int)sizeof(path))
                    throw Error(1, "iteration output path is too long");
                e->read_plane(PLANE_ESTIMATE, 0, plane.data(), 0);
                FILE *f = fopen(path, "wb");
                if (!f) throw Error(1, "cannot create iteration output");
                if (fwrite(plane.data(), sizeof(float), nout, f) != nout) { fclose(f); throw Error(1, "iteration output write failed"); }
                if (fclose(f)) throw Error(1, "iteration output close failed");
                printf("UPDC iteration %d raw output: %s\n", it, path);
            }
            iter_output[it - 1] = wall() - t1;
            iter_total[it - 1] = wall() - t0;
            printf("UPDC iteration %d/%d: signed sum %.9g, negative %llu/%zu, frozen +%llu total %llu, min raw mu %.9g, "
                   "wall %.3f s [device %.6f]%s\n",
                   it, iterations, r[0].signed_sum, (unsigned long long)r[0].negative, nout, (unsigned long long)nn,
                   (unsigned long long)nt, (double)(float)mn, iter_total[it - 1], r[0].seconds, save ? " SAVE" : "");
            fflush(stdout);
            recs.push_back(r[0]);
        }
        if (fclose(freeze)) throw Error(1, "freeze CSV close failed");
        // WHT = coverage * weight_scale (updc_core.c:1482-1485)
        e->read_plane(PLANE_COVERAGE, 0, plane.data(), 0);
        const float ws = (float)e->scalar(0);
        for (size_t t = 0; t < nout; ++t) plane[t] *= ws;
        FILE *f = fopen(weight_output, "wb");
        if (!f) throw Error(1, "cannot create WHT output");
        if (fwrite(plane.data(), sizeof(float), nout, f) != nout) { fclose(f); throw Error(1, "WHT output write failed"); }
        if (fclose(f)) throw Error(1, "WHT output close failed");
        // timing CSV with the reference's row names (updc_core.c:1487-1508)
        FILE *tf = fopen((prefix + "_timing.csv").c_str(), "w");
        if (!tf) throw Error(1, "cannot write timing CSV");
        fprintf(tf, "stage,wall_seconds\nfft_autotune,%.6f\nfft_plan,%.6f\npsf_cache,%.6f\npolygon_links,%.6f\n"
                    "persistent_mmap,%.6f\nmmap_prewarm,%.6f\ndata_cache,%.6f\nweight_scale,%.6f\ninitial_drizzle,%.6f\n"
                    "sensitivity,%.6f\n",
                e->scalar(7), 0.0, e->setup_seconds(2), e->setup_seconds(0), 0.0, 0.0, e->setup_seconds(1), 0.0,
                e->setup_seconds(3), e->setup_seconds(4));
        for (int i = 0; i < iterations; ++i) {
            const IterationRecord &r = recs[i];
            fprintf(tf, "iteration_%02d_estimate_fft,%.6f\n", i + 1, r.stage_seconds[0]);
            fprintf(tf, "iteration_%02d_fused_exposure_wall,%.6f\n", i + 1, r.stage_seconds[1] + r.stage_seconds[2] + r.stage_seconds[3] + r.stage_seconds[4] + r.stage_seconds[5]);
            fprintf(tf, "iteration_%02d_forward_ifft_critical,%.6f\n", i + 1, r.stage_seconds[1] + r.stage_seconds[2]);
            fprintf(tf, "iteration_%02d_fused_detector_critical,%.6f\n", i + 1, r.stage_seconds[3] + r.stage_seconds[4]);
            fprintf(tf, "iteration_%02d_scatter_fft_critical,%.6f\n", i + 1, r.stage_seconds[5]);
            fprintf(tf, "iteration_%02d_adjoint_reduce_ifft,%.6f\n", i + 1, r.stage_seconds[6]);
            fprintf(tf, "iteration_%02d_update,%.6f\n", i + 1, r.stage_seconds[7]);
            fprintf(tf, "iteration_%02d_output,%.6f\n", i + 1, iter_output[i]);
            fprintf(tf, "iteration_%02d_total,%.6f\n", i + 1, r.seconds);
        }
        fprintf(tf, "total_solver,%.6f\n", wall() - total_start);
        if (fclose(tf)) throw Error(1, "timing CSV close failed");
        printf("Setup %.3f s; device memory %.3f GiB\n", setup_time, (double)e->device_bytes() / 1073741824.0);
        struct rusage usage;
        if (!getrusage(RUSAGE_SELF, &usage)) printf("Peak process RSS: %.3f GiB\n", (double)usage.ru_maxrss / 1048576.0);
        fflush(stdout);
    });
}

void UPDC_ALL(const char *manifest, int width, int height, int input_width, int input_height, int exposures,
              int transpose_psf, int iterations, const char *iter_prefix, const char *weight_output,
              int fft_worker_count, int exposure_worker_count, int preprocess_worker_count, int plan_measure,
              int autotune, int retune_fft, const char *wisdom_path, int save_every_arg) {
    if (updc_all(manifest, width, height, input_width, input_height, exposures, transpose_psf, iterations,
                 iter_prefix, weight_output, fft_worker_count, exposure_worker_count, preprocess_worker_count,
                 plan_measure, autotune, retune_fft, wisdom_path, save_every_arg)) {
        fflush(stdout);
        fprintf(stderr, "UPDC_ALL: %s\n", updc_last_error());
        exit(EXIT_FAILURE);
    }
}

}  // extern "C"
