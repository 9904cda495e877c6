// UPDC solver engine: setup stages and the per-iteration kernel sequence.
#include <cub/cub.cuh>

#include <algorithm>
#include <functional>
#include <type_traits>
#include <map>
#include <unistd.h>
#include <chrono>
#include <cmath>
#include <cstring>

#include "engine.cuh"
#include "fft.cuh"
#include "kernels.cuh"
#include "kernels_ct.cuh"
#include "longrow.cuh"
#include "linkmap.cuh"
#include "pointwise.cuh"
#include "nll.cuh"

namespace updc {

void make_tensor_map_3d(CUtensorMap *map, const void *base, uint64_t dim0, uint64_t dim1, uint64_t dim2,
                        uint32_t box0, uint32_t box1) {
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        UPDC_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess) throw Error(-2, "cuTensorMapEncodeTiled is unavailable");
        encode = (Encode)fn;
    }
    // the layout rules of tiled TMA copies, checked before the driver sees them
    if (((uintptr_t)base & 15) || (dim0 * 8) % 16 || (box0 * 8) % 16 || box0 > 256 || box1 > 256 || box0 > dim0)
        throw Error(-2, "tensor map layout violates TMA alignment rules");
    const cuuint64_t dims[3] = {dim0, dim1, dim2};
    const cuuint64_t strides[2] = {dim0 * 8, dim0 * dim1 * 8};
    const cuuint32_t box[3] = {box0, box1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(-2, "cuTensorMapEncodeTiled failed with status " + std::to_string((int)r));
}

const char *error_message(uint32_t code) {
    switch (code) {
        case ERR_NONFINITE_MEAN: return "non-finite forward mean";
        case ERR_NONFINITE_RATIO: return "non-finite y/raw_mu ratio";
        case ERR_NONFINITE_CORRECTION: return "non-finite multiplicative correction";
        case ERR_NEGATIVE_CORRECTION: return "substantially negative multiplicative correction";
        case ERR_NONFINITE_ESTIMATE: return "non-finite signed UPDC estimate";
        case ERR_INVALID_NORM_WHT: return "invalid normalized WHT";
        case ERR_NEGATIVE_YEFF: return "negative/non-finite y_eff reached solver";
        case ERR_NONFINITE_INITIAL: return "non-finite signed initial estimate";
        case ERR_INVALID_PSF_PIXEL: return "invalid PSF pixel";
        case ERR_LINKMAP_TARGET: return "invalid or obsolete LinkMap cache";
        case ERR_DEVICE_TIMEOUT: return "device wait timed out";
        default: return "unknown device error";
    }
}

int next_smooth(int n, bool even) {
    for (;; ++n) {
        if (even && (n & 1)) continue;
        int q = n;
        while (q % 2 == 0) q /= 2;
        while (q % 3 == 0) q /= 3;
        while (q % 5 == 0) q /= 5;
        while (q % 7 == 0) q /= 7;
        if (q == 1) return n;
    }
}

bool fft_factor(int n, int rmax, std::vector<int> &radices) {
    // candidate radices in the order the device stage loops run them
    static const int order[] = {32, 28, 27, 25, 24, 21, 20, 18, 16, 15, 14, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2};
    radices.clear();
    int m = n;
    while (m > 1) {
        int pick = 0;
        for (int r : order)
            if (r <= rmax && m % r == 0) { pick = r; break; }
        if (!pick) return false;
        radices.push_back(pick);
        m /= pick;
    }
    std::vector<int> sorted;
    for (int r : order)
        for (int x : radices)
            if (x == r) sorted.push_back(x);
    radices = sorted;
    return (int)radices.size() <= FFT_MAX_STAGES;
}

void fft_factorizations(int n, int rmax, int extra_stages, std::vector<std::vector<int>> &out) {
    static const int order[] = {32, 28, 27, 25, 24, 21, 20, 18, 16, 15, 14, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2};
    out.clear();
    std::vector<int> greedy;
    if (!fft_factor(n, rmax, greedy)) return;
    const int max_stages = (int)greedy.size() + extra_stages;
    // depth-first over non-increasing radix sequences (the device's stage order)
    std::vector<int> cur;
    std::function<void(int, int)> rec = [&](int m, int first) {
        if (m == 1) {
            if (!cur.empty()) out.push_back(cur);
            return;
        }
        if ((int)cur.size() >= max_stages) return;
        for (int i = first; i < (int)(sizeof(order) / sizeof(order[0])); ++i) {
            const int r = order[i];
            if (r > rmax || m % r) continue;
            cur.push_back(r);
            rec(m / r, i);
            cur.pop_back();
        }
    };
    rec(n, 0);
    if (out.empty()) out.push_back(greedy);
}

template <typename T> std::vector<cx<T>> fft_make_table(int n, const std::vector<int> &rad, FftPlan &plan) {
    long prod = 1;
    for (int r : rad) prod *= r;
    if (prod != n || rad.empty() || (int)rad.size() > FFT_MAX_STAGES)
        throw Error(1, "FFT factorization does not match length " + std::to_string(n));
    std::vector<cx<T>> tab;
    plan = FftPlan();
    plan.n = n;
    plan.nstage = (int)rad.size();
    int ns = 1;
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t s = 0; s < rad.size(); ++s) {
        const int R = rad[s];
        plan.radix[s] = R;
        plan.ns[s] = ns;
        plan.twoff[s] = (int)tab.size();
        plan.ns_div[s] = FastDiv((uint32_t)ns);
        plan.nb_div[s] = FastDiv((uint32_t)(n / R));
        // r-major: the twiddles of input r for consecutive k are adjacent, so
        // the lanes of a warp (consecutive k) load them coalesced
        for (int r = 1; r < R; ++r)
            for (int k = 0; k < ns; ++k) {
                const double a = -two_pi * (double)r * (double)k / ((double)ns * (double)R);
                tab.push_back(cx<T>{(T)std::cos(a), (T)std::sin(a)});
            }
        ns *= R;
    }
    if (tab.empty()) tab.push_back(cx<T>{1, 0});
    return tab;
}

template <typename T> std::vector<cx<T>> fft_make_table(int n, int rmax, FftPlan &plan) {
    std::vector<int> rad;
    if (!fft_factor(n, rmax, rad)) throw Error(1, "FFT length " + std::to_string(n) + " is not 7-smooth");
    return fft_make_table<T>(n, rad, plan);
}
template std::vector<cx<float>> fft_make_table<float>(int, int, FftPlan &);
template std::vector<cx<double>> fft_make_table<double>(int, int, FftPlan &);
template std::vector<cx<float>> fft_make_table<float>(int, const std::vector<int> &, FftPlan &);
template std::vector<cx<double>> fft_make_table<double>(int, const std::vector<int> &, FftPlan &);

namespace {
// Output slot of register p in the codelet of radix R (Dft<R>::out).
int codelet_out(int R, int p) {
    static const int split[][3] = {{6, 2, 3}, {9, 3, 3}, {10, 2, 5}, {12, 4, 3}, {14, 2, 7}, {15, 3, 5}, {16, 4, 4},
                                   {18, 2, 9}, {20, 4, 5}, {21, 3, 7}, {24, 8, 3}, {25, 5, 5}, {27, 3, 9}, {28, 4, 7},
                                   {32, 4, 8}};
    for (const auto &sp : split)
        if (sp[0] == R) return p / sp[2] + sp[1] * codelet_out(sp[2], p % sp[2]);
    return p;
}
// Shared-memory wavefronts of one warp access of 8-byte elements: two
// half-warp phases, each costing the largest number of distinct addresses in
// one bank pair.
int warp_wavefronts(const int *addr, int shift) {
    int total = 0;
    for (int h = 0; h < 2; ++h) {
        int slots[16][16];
        int cnt[16] = {0};
        for (int l = 16 * h; l < 16 * h + 16; ++l) {
            if (addr[l] < 0) continue;
            const int a = fpad(addr[l], shift), b = a & 15;
            bool seen = false;
            for (int i = 0; i < cnt[b]; ++i) seen |= slots[b][i] == a;
            if (!seen) slots[b][cnt[b]++] = a;
        }
        int mx = 0;
        for (int b = 0; b < 16; ++b) mx = std::max(mx, cnt[b]);
        total += mx;
    }
    return total;
}
}  // namespace

int fft_choose_padding(const FftPlan &plan, int nt, int cap, int batch) {
    int best_shift = 31;
    long best = -1;
    for (int shift : {31, 5, 4}) {
        long cost = 0;
        const int n = plan.n;
        for (int s = 0; s < plan.nstage; ++s) {
            const int R = plan.radix[s], Ns = plan.ns[s], nb = n / R, total = nb * batch;
            const int K = (cap / R + nt - 1) / nt;
            int addr[32];
            for (int kk = 0; kk < K; ++kk)
                for (int w = 0; w < nt / 32; ++w) {
                    if (w * 32 + kk * nt >= total) break;
                    for (int r = 0; r < R; ++r) {
                        for (int l = 0; l < 32; ++l) {
                            const int b = w * 32 + l + kk * nt;
                            addr[l] = b < total ? (b / nb) * n + b % nb + r * nb : -1;
                        }
                        cost += warp_wavefronts(addr, shift);
                        for (int l = 0; l < 32; ++l) {
                            const int b = w * 32 + l + kk * nt;
                            if (b >= total) { addr[l] = -1; continue; }
                            const int row = b / nb, j = b % nb, k = j % Ns;
                            addr[l] = row * n + (j - k) * R + k + codelet_out(R, r) * Ns;
                        }
                        cost += warp_wavefronts(addr, shift);
                    }
                }
        }
        if (best < 0 || cost < best) {
            best = cost;
            best_shift = shift;
        }
    }
    return best_shift;
}

namespace {

constexpr int NT = SPEC_NT;
template <typename T> using NtAdj = SpecNtAdj<T>;
template <typename T> using ColNt = SpecColNt<T>;
template <typename T> using RowNt = SpecRowNt<T>;
// FP32 column kernels always keep X-hat and the accumulator in global scratch
template <typename T> constexpr int ColAux = sizeof(T) == 4 ? 1 : 0;
// Runs f with the plan's padding shift as a compile-time constant where the
// kernels are compiled for it (31: no padding, every fpad() folds away),
// else with -1 (the kernels read it from the plan).
template <class F> void by_pad(int sh, F &&f) {
    if (sh == 31) f(std::integral_constant<int, 31>{});
    else f(std::integral_constant<int, -1>{});
}
// Same for the rows of a row tile (2, the usual FP32 tile, or read at run time).
template <class F> void by_rows(int b, F &&f) {
    if (b == 2) f(std::integral_constant<int, 2>{});
    else f(std::integral_constant<int, 0>{});
}
template <typename T> using Caps = SpecCaps<T>;
constexpr size_t SMEM_LIMIT = SPEC_SMEM_LIMIT;

template <typename T> T *dalloc(size_t n, size_t *counter) {
    T *p = nullptr;
    UPDC_CUDA(cudaMalloc(&p, (n ? n : 1) * sizeof(T)));
    if (counter) *counter += (n ? n : 1) * sizeof(T);
    return p;
}

int grid1d(size_t n, int threads = 256) {
    size_t g = (n + threads - 1) / threads;
    if (g > 148 * 16) g = 148 * 16;
    return (int)(g ? g : 1);
}

template <typename K> void set_smem(K kern, size_t bytes) { raise_smem_limit(reinterpret_cast<const void *>(kern), bytes); }

size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool read_f32_exact(const std::string &path, float *out, size_t count) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    const bool ok = fread(out, sizeof(float), count, f) == count && fgetc(f) == EOF;
    fclose(f);
    return ok;
}

// ---------------------------------------------------------------------------- engine
template <typename T> class EngineImpl final : public Engine {
  public:
    explicit EngineImpl(const EngineOptions &o) : opt_(o) {
        UPDC_CUDA(cudaSetDevice(opt_.device));
        UPDC_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        comp_mu_ = opt_.compensated_mu >= 0 ? opt_.compensated_mu
                                            : (opt_.form == FORM_FP32 || opt_.form == FORM_FP32_KAHAN ? 1 : 0);
    }
    ~EngineImpl() override {
        drop_loop_graphs();
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (graph_) cudaGraphDestroy(graph_);
        for (auto &m : links_) m.release();
        for (void *p : allocs_) cudaFree(p);
        if (staging_) cudaFree(staging_);
        if (d_psf_grad_) cudaFree(d_psf_grad_);
        if (pinned_) cudaFreeHost(pinned_);
        for (auto e : events_) cudaEventDestroy(e);
        if (stream_) cudaStreamDestroy(stream_);
    }

    // ------------------------------------------------------------------ load
    void load(const std::string &manifest, int W, int H, int iw, int ih, int nexp, int transposed) override {
        if (W < 1 || H < 1 || iw < 1 || ih < 1 || nexp < 1) throw Error(1, "invalid dimensions/exposures/iterations/workers/save_every");
        W_ = W; H_ = H; iw_ = iw; ih_ = ih; nexp_ = nexp; transposed_ = transposed ? 1 : 0;
        nout_ = (size_t)W * H;
        nin_ = (size_t)iw * ih;
        if (nout_ > UINT32_MAX) throw Error(1, "target grid exceeds 32-bit link index capacity");
        FILE *f = fopen(manifest.c_str(), "r");
        if (!f) throw Error(1, "cannot open manifest");
        exps_.assign(nexp, ExposureInput());
        for (int k = 0; k < nexp; ++k) {
            char line[8192];
            if (!fgets(line, sizeof(line), f)) { fclose(f); throw Error(1, "manifest has fewer rows than expected"); }
            char *save = nullptr, *fld[8];
            for (int j = 0; j < 8; ++j) fld[j] = strtok_r(j ? nullptr : line, "\t\r\n", &save);
            for (int j = 0; j < 8; ++j)
                if (!fld[j]) { fclose(f); throw Error(1, "manifest requires science, weight, psf, psf_width, psf_height, vertices, background, pedestal"); }
            ExposureInput &e = exps_[k];
            e.science = fld[0]; e.weight = fld[1]; e.psf = fld[2];
            e.psf_width = (int)strtol(fld[3], nullptr, 10);
            e.psf_height = (int)strtol(fld[4], nullptr, 10);
            e.vertices = fld[5];
            e.links = e.vertices + ".links";
            e.background = strtod(fld[6], nullptr);
            e.pedestal = strtod(fld[7], nullptr);
            e.backgroundf = strtof(fld[6], nullptr);
            e.pedestalf = strtof(fld[7], nullptr);
            if (e.psf_width < 1 || e.psf_height < 1) { fclose(f); throw Error(1, "invalid PSF dimensions in manifest"); }
            const float mo = e.backgroundf + e.pedestalf;
            if (!std::isfinite(e.backgroundf) || !std::isfinite(e.pedestalf) || e.pedestalf < 0.0f || !std::isfinite(mo)) {
                fclose(f);
                throw Error(1, "invalid background/pedestal in manifest");
            }
        }
        char extra[8192];
        const bool more = fgets(extra, sizeof(extra), f) != nullptr;
        fclose(f);
        if (more) throw Error(1, "manifest has more rows than expected");
    }

    // ------------------------------------------------------------------ setup
    void setup() override {
        const double t_all = now_s();
        choose_fft_shape();
        allocate();
        double t0 = now_s();
        for (int k = 0; k < nexp_; ++k)
            if (active(k)) prepare_links(k);
        setup_time_[0] = now_s() - t0;
        t0 = now_s();
        load_planes();
        setup_time_[1] = now_s() - t0;
        t0 = now_s();
        prepare_psf_spectra();
        setup_time_[2] = now_s() - t0;
        t0 = now_s();
        drizzle();
        setup_time_[3] = now_s() - t0;
        t0 = now_s();
        denominator();
        setup_time_[4] = now_s() - t0;
        setup_time_[5] = now_s() - t_all;
        // an exposure shard set up alone waits for its partial planes to be
        // summed over the shards (finish_shard_setup)
        setup_done_ = !shard_setup_;
        shard_setup_pending_ = shard_setup_;
    }

    void iterate(int n, bool check_each, std::vector<IterationRecord> *records) override {
        if (!setup_done_) throw Error(1, "engine is not set up");
        const bool graph = opt_.use_graph && !opt_.stage_timing;
        if (graph && !graph_exec_) build_graph();
        while ((int)events_.size() < 2 * (n + 1)) {
            cudaEvent_t e;
            UPDC_CUDA(cudaEventCreate(&e));
            events_.push_back(e);
        }
        const size_t rec_bytes = rec_stride();
        ensure_pinned((size_t)n * rec_bytes);
        // without per-iteration checks the whole loop of n iterations is one
        // CUDA graph (iterations, their events and record copies)
        const bool whole = graph && !check_each && n > 1 && n <= LOOP_GRAPH_MAX;
        int done = 0;
        while (done < n) {
            const int batch = check_each ? 1 : n - done;
            if (whole) {
                UPDC_CUDA(cudaGraphLaunch(loop_graph(n), stream_));
            } else {
                for (int i = 0; i < batch; ++i) enqueue_recorded(done + i, graph);
            }
            UPDC_CUDA(cudaStreamSynchronize(stream_));
            for (int i = 0; i < batch; ++i) {
                const char *src = (const char *)pinned_ + (size_t)(done + i) * rec_bytes;
                unsigned long long key;
                memcpy(&key, src + nexp_ * sizeof(ExpStats), 8);
                if (key != ~0ull) raise_device_error(key);
                if (records) {
                    IterationRecord r;
                    float ms = 0;
                    UPDC_CUDA(cudaEventElapsedTime(&ms, events_[2 * (done + i)], events_[2 * (done + i) + 1]));
                    r.seconds = ms * 1e-3;
                    if (opt_.stage_timing)
                        for (int s = 0; s < 8; ++s) r.stage_seconds[s] = stage_ms_[s] * 1e-3;
                    const ExpStats *st = (const ExpStats *)src;
                    for (int k = 0; k < nexp_; ++k) {
                        r.new_frozen.push_back(st[k].nnew);
                        r.total_frozen.push_back(st[k].ntotal);
                        r.min_raw_mu.push_back(st[k].min_ordered == ~0ull ? INFINITY : ordered_to_double(st[k].min_ordered));
                    }
                    memcpy(&r.signed_sum, src + nexp_ * sizeof(ExpStats) + 8, 8);
                    memcpy(&r.negative, src + nexp_ * sizeof(ExpStats) + 16, 8);
                    records->push_back(std::move(r));
                }
            }
            done += batch;
        }
    }

    // ------------------------------------------------------------------ planes
    // Host <-> device plane copies on the engine's stream.  When the host type
    // is the engine's type the copy is direct (pinned host memory gives full
    // PCIe/C2C bandwidth); otherwise the raw host data goes through a device
    // staging buffer and is converted by a kernel.
    void read_plane(int which, int k, void *host, int as_double) override {
        size_t n;
        const void *src = plane_ptr(which, k, &n);
        if (which == PLANE_FROZEN) {
            UPDC_CUDA(cudaMemcpyAsync(host, src, n, cudaMemcpyDeviceToHost, stream_));
        } else if ((as_double != 0) == (sizeof(T) == 8)) {
            UPDC_CUDA(cudaMemcpyAsync(host, src, n * sizeof(T), cudaMemcpyDeviceToHost, stream_));
        } else {
            void *st = staging(n * 8);
            if (as_double) k_convert<T, double><<<grid1d(n), 256, 0, stream_>>>((const T *)src, (double *)st, n);
            else k_convert<T, float><<<grid1d(n), 256, 0, stream_>>>((const T *)src, (float *)st, n);
            UPDC_CUDA(cudaGetLastError());
            UPDC_CUDA(cudaMemcpyAsync(host, st, n * (as_double ? 8 : 4), cudaMemcpyDeviceToHost, stream_));
        }
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }
    void write_plane(int which, int k, const void *host, int as_double) override {
        size_t n;
        void *dst = const_cast<void *>(plane_ptr(which, k, &n));
        if (which == PLANE_FROZEN) {
            UPDC_CUDA(cudaMemcpyAsync(dst, host, n, cudaMemcpyHostToDevice, stream_));
        } else if ((as_double != 0) == (sizeof(T) == 8)) {
            UPDC_CUDA(cudaMemcpyAsync(dst, host, n * sizeof(T), cudaMemcpyHostToDevice, stream_));
        } else {
            void *st = staging(n * 8);
            UPDC_CUDA(cudaMemcpyAsync(st, host, n * (as_double ? 8 : 4), cudaMemcpyHostToDevice, stream_));
            if (as_double) k_convert<double, T><<<grid1d(n), 256, 0, stream_>>>((const double *)st, (T *)dst, n);
            else k_convert<float, T><<<grid1d(n), 256, 0, stream_>>>((const float *)st, (T *)dst, n);
            UPDC_CUDA(cudaGetLastError());
        }
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }
    void *staging(size_t bytes) {
        if (bytes > staging_bytes_) {
            if (staging_) cudaFree(staging_);
            staging_ = nullptr;
            UPDC_CUDA(cudaMalloc(&staging_, bytes));
            staging_bytes_ = bytes;
        }
        return staging_;
    }
    void *staging_ = nullptr;
    size_t staging_bytes_ = 0;

    void stage_forward(int k) override {
        (void)k;
        reset_iteration_state();
        launch_row_r2c_plane(estimate_, rx_, 1, 0, map_rx_);
        launch_col_forward();
        launch_row_c2r_batched(act_y(), act_n_, blur_ + (size_t)act_k0_ * nout_, map_y_);
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }
    void stage_detector(int k, IterationRecord *rec) override {
        reset_iteration_state();
        launch_detector();
        launch_scatter(wr_, scatter_);
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        check_error();
        if (rec) {
            std::vector<ExpStats> st(nexp_);
            UPDC_CUDA(cudaMemcpy(st.data(), d_stats_, nexp_ * sizeof(ExpStats), cudaMemcpyDeviceToHost));
            rec->new_frozen.clear(); rec->total_frozen.clear(); rec->min_raw_mu.clear();
            for (int j = 0; j < nexp_; ++j) {
                rec->new_frozen.push_back(st[j].nnew);
                rec->total_frozen.push_back(st[j].ntotal);
                rec->min_raw_mu.push_back(st[j].min_ordered == ~0ull ? INFINITY : ordered_to_double(st[j].min_ordered));
            }
        }
        (void)k;
    }
    void stage_correction() override {
        launch_row_r2c_plane(scatter_ + (size_t)act_k0_ * nout_, act_rs(), act_n_, nout_, map_rs_);
        launch_col_adjoint();
        launch_row_c2r_batched(cr_, 1, correction_, map_cr_);
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }
    void *plane_device(int which) override {
        switch (which) {
            case PLANE_ESTIMATE: return estimate_;
            case PLANE_COVERAGE: return coverage_;
            case PLANE_DENOMINATOR: return den_;
            case PLANE_CORRECTION: return correction_;
            default: throw Error(1, "plane has no single device address");
        }
    }
    cudaStream_t stream() const override { return stream_; }
    void enqueue_partial() override { enqueue_stages([](int) {}, false); }
    void enqueue_update() override { launch_update(); }
    void finish_iteration(IterationRecord *rec) override {
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        check_error();
        if (!rec) return;
        std::vector<ExpStats> st(nexp_);
        UPDC_CUDA(cudaMemcpy(st.data(), d_stats_, nexp_ * sizeof(ExpStats), cudaMemcpyDeviceToHost));
        rec->new_frozen.clear(); rec->total_frozen.clear(); rec->min_raw_mu.clear();
        for (int j = 0; j < nexp_; ++j) {
            rec->new_frozen.push_back(st[j].nnew);
            rec->total_frozen.push_back(st[j].ntotal);
            rec->min_raw_mu.push_back(st[j].min_ordered == ~0ull ? INFINITY : ordered_to_double(st[j].min_ordered));
        }
        UPDC_CUDA(cudaMemcpy(&rec->signed_sum, d_red_sum_, 8, cudaMemcpyDeviceToHost));
        UPDC_CUDA(cudaMemcpy(&rec->negative, d_red_neg_, 8, cudaMemcpyDeviceToHost));
    }
    void stage_update(IterationRecord *rec) override {
        reset_iteration_state();
        launch_update();
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        check_error();
        if (rec) {
            UPDC_CUDA(cudaMemcpy(&rec->signed_sum, d_red_sum_, 8, cudaMemcpyDeviceToHost));
            UPDC_CUDA(cudaMemcpy(&rec->negative, d_red_neg_, 8, cudaMemcpyDeviceToHost));
        }
    }
    // Exposures [act_k0_, act_k0_ + act_n_) take part in the iterations
    // (all by default; an exposure shard of a multi-GPU solve otherwise).
    int act_k0_ = 0, act_n_ = 0;
    cx<T> *act_y() const { return y_ + (size_t)act_k0_ * ((size_t)M_ + 1) * ldh_; }
    cx<T> *act_rs() const { return rs_ + (size_t)act_k0_ * ((size_t)M_ + 1) * ldh_; }
    void build_exposure_maps() {
        if (!use_tma_) return;
        constexpr int EW = TmaElems<T>::value;
        const uint64_t d0 = (uint64_t)ldh_ * EW;
        const uint32_t ub = (uint32_t)row_ubox(M_);
        make_tensor_map_3d(&map_y_, act_y(), d0, (uint64_t)M_ + 1, act_n_, row_b_ * EW, ub);
        make_tensor_map_3d(&map_rs_, act_rs(), d0, (uint64_t)M_ + 1, act_n_, row_b_ * EW, ub);
    }
    void set_active_exposures(int k0, int n) override {
        if (k0 < 0 || n < 1 || k0 + n > nexp_) throw Error(1, "active exposure range out of bounds");
        if (!setup_done_) {
            // before setup: set up this exposure shard alone (see setup)
            if (shard_setup_pending_) throw Error(1, "shard setup is waiting for finish_shard_setup");
            act_k0_ = k0;
            act_n_ = n;
            shard_setup_ = n < nexp_;
            return;
        }
        act_k0_ = k0;
        act_n_ = n;
        build_exposure_maps();
        drop_loop_graphs();
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (graph_) cudaGraphDestroy(graph_);
        graph_exec_ = nullptr;
        graph_ = nullptr;
    }
    void refresh_sensitivity() override { finish_denominator(); }
    // Shard setup: only exposures [act_k0_, act_k0_ + act_n_) get LinkMaps
    // and PSF spectra, and the drizzle and denominator leave partial planes
    // (COVERAGE, ESTIMATE = the data sum, CORRECTION = the background sum,
    // DENOMINATOR) for the caller to sum over the shards.
    bool shard_setup_ = false, shard_setup_pending_ = false;
    bool active(int k) const { return !shard_setup_ || (k >= act_k0_ && k < act_k0_ + act_n_); }
    void finish_shard_setup() override {
        if (!shard_setup_pending_) throw Error(1, "no shard setup is waiting for its sums");
        UPDC_CUDA(cudaMemset(d_err_, 0xFF, 8));
        k_drizzle_finish<T><<<grid1d(nout_), 256, 0, stream_>>>(nout_, coverage_, estimate_, correction_, estimate_, d_err_);
        UPDC_CUDA(cudaGetLastError());
        UPDC_CUDA(cudaMemsetAsync(correction_, 0, nout_ * sizeof(T), stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        check_error();
        finish_denominator();
        shard_setup_pending_ = false;
        setup_done_ = true;
    }

    // ------------------------------------------------------------------ checkpoint / resume
    // State file: a 64-byte header {"UPDCSTAT", u32 version 1, u32 element
    // bytes, u32 W, H, iw, ih, nexp, u32 0, u64 iteration, u64 0 x 2}, the
    // estimate (W*H elements of the engine's precision) and the persistent
    // FreezeMu masks (nexp*iw*ih bytes): everything the next iteration
    // depends on besides the set-up products, which are rebuilt from the
    // manifest.  Written to a temporary name and renamed into place.
    void save_state(const std::string &path, uint64_t iteration) override {
        if (!setup_done_) throw Error(1, "engine is not set up");
        std::vector<T> x(nout_);
        std::vector<uint8_t> fz(nexp_ * nin_);
        UPDC_CUDA(cudaMemcpyAsync(x.data(), estimate_, nout_ * sizeof(T), cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaMemcpyAsync(fz.data(), frozen_, fz.size(), cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        unsigned char hdr[64] = {};
        memcpy(hdr, "UPDCSTAT", 8);
        const uint32_t f[8] = {1u, (uint32_t)sizeof(T), (uint32_t)W_, (uint32_t)H_, (uint32_t)iw_, (uint32_t)ih_,
                               (uint32_t)nexp_, 0u};
        memcpy(hdr + 8, f, sizeof(f));
        memcpy(hdr + 40, &iteration, 8);
        const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
        FILE *o = fopen(tmp.c_str(), "wb");
        if (!o) throw Error(1, "cannot create state file: " + path);
        const bool ok = fwrite(hdr, 1, 64, o) == 64 && fwrite(x.data(), sizeof(T), nout_, o) == nout_ &&
                        fwrite(fz.data(), 1, fz.size(), o) == fz.size();
        if (fclose(o) || !ok || rename(tmp.c_str(), path.c_str())) {
            unlink(tmp.c_str());
            throw Error(1, "state file write failed: " + path);
        }
    }
    void load_state(const std::string &path, uint64_t *iteration) override {
        if (!setup_done_) throw Error(1, "engine is not set up");
        FILE *in = fopen(path.c_str(), "rb");
        if (!in) throw Error(1, "cannot open state file: " + path);
        unsigned char hdr[64];
        uint32_t f[8];
        std::vector<T> x(nout_);
        std::vector<uint8_t> fz(nexp_ * nin_);
        bool ok = fread(hdr, 1, 64, in) == 64 && memcmp(hdr, "UPDCSTAT", 8) == 0;
        if (ok) {
            memcpy(f, hdr + 8, sizeof(f));
            ok = f[0] == 1u && f[1] == sizeof(T) && f[2] == (uint32_t)W_ && f[3] == (uint32_t)H_ &&
                 f[4] == (uint32_t)iw_ && f[5] == (uint32_t)ih_ && f[6] == (uint32_t)nexp_;
        }
        ok = ok && fread(x.data(), sizeof(T), nout_, in) == nout_ && fread(fz.data(), 1, fz.size(), in) == fz.size();
        char extra;
        ok = ok && fread(&extra, 1, 1, in) == 0;
        fclose(in);
        if (!ok) throw Error(1, "state file does not match this field and precision: " + path);
        if (iteration) memcpy(iteration, hdr + 40, 8);
        UPDC_CUDA(cudaMemcpyAsync(estimate_, x.data(), nout_ * sizeof(T), cudaMemcpyHostToDevice, stream_));
        UPDC_CUDA(cudaMemcpyAsync(frozen_, fz.data(), fz.size(), cudaMemcpyHostToDevice, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }

    FieldView field_view() const override {
        if (!setup_done_) throw Error(1, "engine is not set up");
        if (long_rows_ || long_cols_) throw Error(1, "batched fields need FFT shapes within the one-block transform capacity");
        FieldView v;
        v.elem_bytes = sizeof(T);
        v.form = opt_.form;
        v.comp_mu = comp_mu_;
        v.W = W_, v.H = H_, v.M = M_, v.FH = FH_, v.ldh = ldh_, v.row_b = wide_rows_ ? 1 : row_b_, v.nexp = nexp_;
        v.upd_grid = upd_grid_;
        v.nin = nin_, v.nout = nout_;
        v.plan_m = plan_m_, v.plan_h = plan_h_;
        v.scale = (double)scale_factor();
        v.max_sens = (double)max_sens_;
        v.post = post_;
        v.estimate = estimate_, v.den = den_, v.correction = correction_, v.blur = blur_, v.scatter = scatter_, v.wr = wr_;
        v.rx = rx_, v.y = y_, v.rs = rs_, v.cr = cr_, v.khat = khat_;
        // the batched column kernels keep X-hat and the accumulator in shared memory
        const size_t fb = fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift);
        size_t accb = sizeof(cx<T>);
        if (sizeof(T) == 4 && opt_.form == FORM_FP32) accb = sizeof(AccF64::S);
        if (sizeof(T) == 4 && opt_.form == FORM_FP32_KAHAN) accb = sizeof(AccKahan::S);
        v.needs_aux = FH_ > Caps<T>::COL_S || fb + align16((size_t)FH_ * sizeof(cx<T>)) > SMEM_LIMIT ||
                      fb + align16((size_t)FH_ * accb) > SMEM_LIMIT;
        v.exps = d_exps_;
        v.stats = d_stats_;
        v.err = d_err_;
        v.part_sum = d_part_sum_, v.part_neg = d_part_neg_, v.red_sum = d_red_sum_, v.red_neg = d_red_neg_;
        return v;
    }

    // ------------------------------------------------------------------ differentiable model
    void set_exposure_offsets(int k, double background, double pedestal) override {
        if (k < 0 || k >= nexp_) throw Error(1, "exposure index out of range");
        if (!std::isfinite(background) || !std::isfinite(pedestal) || pedestal < 0)
            throw Error(1, "invalid background/pedestal");
        ExposureInput &e = exps_[k];
        e.background = background;
        e.pedestal = pedestal;
        e.backgroundf = (float)background;
        e.pedestalf = (float)pedestal;
        upload_descs();
    }
    void set_psf(int k, const void *psf, int pw, int phh, int as_double) override {
        if (k < 0 || k >= nexp_) throw Error(1, "exposure index out of range");
        const int tw = transposed_ ? phh : pw, th = transposed_ ? pw : phh;
        if (pw < 1 || phh < 1 || min_fft_length(W_, tw) > FW_ || min_fft_length(H_, th) > FH_)
            throw Error(1, "PSF larger than the FFT shape allows");
        const size_t nu = (size_t)M_ + 1;
        cx<T> *rp = scratch_spec(0);
        const bool fp64_sum = opt_.form == FORM_FP32 || opt_.form == FORM_FP64;
        if (as_double)
            psf_spectrum_one<T, double>((const double *)psf, pw, phh, khat_ + (size_t)k * nu * FH_, rp, fp64_sum,
                                        plan_m_, plan_h_, post_);
        else
            psf_spectrum_one<T, float>((const float *)psf, pw, phh, khat_ + (size_t)k * nu * FH_, rp, fp64_sum,
                                       plan_m_, plan_h_, post_);
        exps_[k].psf_width = pw;
        exps_[k].psf_height = phh;
    }
    void nll(double *terms) override {
        stage_forward(0);
        const unsigned g = (unsigned)std::min<size_t>(ceil_div(nin_, 256), 148 * 4);
        if (!d_nll_part_) d_nll_part_ = alloc<double>((size_t)g * nexp_ * NLL_TERMS);
        k_nll<T><<<dim3(g, (unsigned)nexp_), 256, 0, stream_>>>(d_exps_, nin_, nout_, blur_, wr_, d_nll_part_);
        UPDC_CUDA(cudaGetLastError());
        std::vector<double> &h = nll_parts_;
        h.assign((size_t)g * nexp_ * NLL_TERMS, 0.0);
        UPDC_CUDA(cudaMemcpyAsync(h.data(), d_nll_part_, h.size() * 8, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        // block partials summed in block order with Neumaier compensation
        for (int k = 0; k < nexp_; ++k)
            for (int i = 0; i < NLL_TERMS; ++i) {
                double t = 0, c = 0;
                for (unsigned b = 0; b < g; ++b) {
                    const double v = h[((size_t)k * g + b) * NLL_TERMS + i], u = t + v;
                    c += std::fabs(t) >= std::fabs(v) ? (t - u) + v : (v - u) + t;
                    t = u;
                }
                terms[k * NLL_TERMS + i] = t + c;
            }
    }
    // Per-block partial sums of the last nll() (nexp x blocks x 4): the
    // difference of two evaluations taken partial by partial is exact where
    // the inputs did not change, which finite differences of single pixels need.
    std::vector<double> nll_parts_;
    const std::vector<double> &nll_partials() const override { return nll_parts_; }
    void nll_adjoint() override {
        launch_scatter(wr_, scatter_);
        stage_correction();
    }
    void psf_gradient(int k, double *out) override {
        if (k < 0 || k >= nexp_) throw Error(1, "exposure index out of range");
        const ExposureInput &e = exps_[k];
        const size_t nu = (size_t)M_ + 1, ns = nu * FH_;
        cx<T> *xs = scratch_spec(0), *as = scratch_spec(1);
        // X = FFT2(pad(x)), A = FFT2(pad(S^T r_k)), both u-major (M+1) x FH
        launch_row_r2c_plane(estimate_, rx_, 1, 0, map_rx_);
        launch_col_fft<false>(rx_, ldh_, H_, xs, FH_, FH_);
        launch_row_r2c_plane(scatter_ + (size_t)k * nout_, act_rs(), 1, 0, map_rs_);
        launch_col_fft<false>(act_rs(), ldh_, H_, as, FH_, FH_);
        // correlation c = IFFT2(A conj(X)) / nf, kept on the PSF window
        k_mul_conj<T><<<grid1d(ns), 256, 0, stream_>>>(as, xs, ns);
        launch_col_fft<true>(as, FH_, FH_, xs, FH_, FH_);
        const size_t count = (size_t)e.psf_width * e.psf_height;
        if (!d_psf_grad_ || psf_grad_count_ < count) {
            if (d_psf_grad_) cudaFree(d_psf_grad_);
            d_psf_grad_ = dalloc<double>(count, nullptr);
            psf_grad_count_ = count;
        }
        UPDC_CUDA(cudaMemsetAsync(d_psf_grad_, 0, count * 8, stream_));
        const int fwid = transposed_ ? e.psf_height : e.psf_width, fhei = transposed_ ? e.psf_width : e.psf_height;
        const PsfWindowStore<T> epi{d_psf_grad_, e.psf_width, fwid, fhei, FW_, FH_, transposed_};
        if (long_rows_) {
            long_c2r<T>(lrp_, post_, SpecRef{xs, FH_, 0}, FH_, 1, FW_, (T)(1.0 / ((double)FW_ * (double)FH_)), epi,
                        long_scratch_);
            UPDC_CUDA(cudaMemcpyAsync(out, d_psf_grad_, count * 8, cudaMemcpyDeviceToHost, stream_));
            UPDC_CUDA(cudaStreamSynchronize(stream_));
            return;
        }
        const int B = wide_rows_ ? 1 : row_b_;
        const size_t rsm = row_buf_bytes(B, M_, sizeof(cx<T>), plan_m_.pad_shift);
        set_smem(k_row_c2r<T, RowNt<T>::value, Caps<T>::ROW, PsfWindowStore<T>, false>, rsm);
        dim3 grid((unsigned)ceil_div(FH_, B), 1);
        k_row_c2r<T, RowNt<T>::value, Caps<T>::ROW, PsfWindowStore<T>, false><<<grid, RowNt<T>::value, rsm, stream_>>>(
            plan_m_, post_, SpecRef{xs, FH_, 0}, no_map_, FH_, FW_, B, FastDiv((uint32_t)B),
            (T)(1.0 / ((double)FW_ * (double)FH_)), epi, d_err_);
        UPDC_CUDA(cudaGetLastError());
        UPDC_CUDA(cudaMemcpyAsync(out, d_psf_grad_, count * 8, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }
    void copy_plane_device(int which, int k, void *dptr, int to_engine, int as_double, cudaStream_t stream) override {
        if (which == PLANE_FROZEN) throw Error(1, "device copies cover the floating-point planes");
        size_t n;
        void *plane = const_cast<void *>(plane_ptr(which, k, &n));
        // order the engine's stream after the caller's
        cudaEvent_t ev;
        UPDC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        UPDC_CUDA(cudaEventRecord(ev, stream));
        UPDC_CUDA(cudaStreamWaitEvent(stream_, ev, 0));
        cudaEventDestroy(ev);
        const bool same = (as_double != 0) == (sizeof(T) == 8);
        if (to_engine) {
            if (same) UPDC_CUDA(cudaMemcpyAsync(plane, dptr, n * sizeof(T), cudaMemcpyDeviceToDevice, stream_));
            else if (as_double) k_convert<double, T><<<grid1d(n), 256, 0, stream_>>>((const double *)dptr, (T *)plane, n);
            else k_convert<float, T><<<grid1d(n), 256, 0, stream_>>>((const float *)dptr, (T *)plane, n);
        } else {
            if (same) UPDC_CUDA(cudaMemcpyAsync(dptr, plane, n * sizeof(T), cudaMemcpyDeviceToDevice, stream_));
            else if (as_double) k_convert<T, double><<<grid1d(n), 256, 0, stream_>>>((const T *)plane, (double *)dptr, n);
            else k_convert<T, float><<<grid1d(n), 256, 0, stream_>>>((const T *)plane, (float *)dptr, n);
        }
        UPDC_CUDA(cudaGetLastError());
        UPDC_CUDA(cudaStreamSynchronize(stream_));
    }
    double *d_nll_part_ = nullptr, *d_psf_grad_ = nullptr;
    size_t psf_grad_count_ = 0;
    cx<T> *scratch_spec_[2] = {nullptr, nullptr};
    // (M+1) x FH complex scratch planes of the differentiable-model paths
    cx<T> *scratch_spec(int i) {
        if (!scratch_spec_[i]) scratch_spec_[i] = alloc<cx<T>>(((size_t)M_ + 1) * FH_);
        return scratch_spec_[i];
    }
    // column transforms of M+1 columns: `in` has `rows_in` rows at pitch ldi
    template <bool INV> void launch_col_fft(const cx<T> *in, int ldi, int rows_in, cx<T> *out, int ldo, int rows_out) {
        const size_t nu = (size_t)M_ + 1;
        if (long_cols_) return long_col_fft<T, INV>(lcp_, in, ldi, rows_in, out, ldo, rows_out, (int)nu, long_col_scratch_);
        const size_t cs = fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift);
        if (FH_ <= Caps<T>::COL_S) {
            set_smem(k_col_fft<T, NT, Caps<T>::COL_S, INV>, cs);
            k_col_fft<T, NT, Caps<T>::COL_S, INV><<<(unsigned)nu, NT, cs, stream_>>>(plan_h_, in, ldi, rows_in, out, ldo, rows_out);
        } else {
            set_smem(k_col_fft<T, NT, Caps<T>::COL_L, INV>, cs);
            k_col_fft<T, NT, Caps<T>::COL_L, INV><<<(unsigned)nu, NT, cs, stream_>>>(plan_h_, in, ldi, rows_in, out, ldo, rows_out);
        }
        UPDC_CUDA(cudaGetLastError());
    }

    void decode_links(int k, uint32_t *host_targets) override {
        const DevLinkMap &m = links_.at(k);
        uint32_t *d = dalloc<uint32_t>(m.nlinks, nullptr);
        linkmap_decode(m, d, stream_);
        UPDC_CUDA(cudaMemcpyAsync(host_targets, d, m.nlinks * 4, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(d);
    }
    uint64_t link_count(int k) const override { return links_.at(k).nlinks; }
    int link_encoding(int k) const override { return (int)links_.at(k).encoding; }
    double scalar(int which) const override {
        switch (which) {
            case 0: return (double)weight_scale_;
            case 1: return (double)max_sens_;
            case 2: return FW_;
            case 3: return FH_;
            case 4: return (double)masked_;
            case 5: return sizeof(T) * 8;
            case 6: return comp_mu_;
            case 7: return choice_.seconds;
            case 8: return choice_.candidates;
            case 9: return choice_.cache_hit ? 1 : 0;
            case 10: return choice_.predicted_ms;
            case 11:
                return (ct_rows() ? 1 : 0) | (ct_cols() ? 2 : 0) | (fused_gather() ? 4 : 0) | (long_rows_ ? 8 : 0) |
                       (long_cols_ ? 16 : 0) | (wide_rows_ ? 32 : 0);
            default: return 0;
        }
    }
    size_t device_bytes() const override { return bytes_; }
    const std::vector<ExposureInput> &exposures() const override { return exps_; }
    double setup_seconds(int stage) const override { return stage >= 0 && stage < 8 ? setup_time_[stage] : 0; }
    void set_stage_timing(int on) override { opt_.stage_timing = on ? 1 : 0; }

  private:
    EngineOptions opt_;
    cudaStream_t stream_ = nullptr;
    int comp_mu_ = 0;
    int W_ = 0, H_ = 0, iw_ = 0, ih_ = 0, nexp_ = 0, transposed_ = 0, FW_ = 0, FH_ = 0, M_ = 0;
    size_t nout_ = 0, nin_ = 0, bytes_ = 0;
    std::vector<ExposureInput> exps_;
    std::vector<DevLinkMap> links_;
    std::vector<void *> allocs_;
    bool setup_done_ = false;
    double setup_time_[8] = {};
    float stage_ms_[8] = {};

    FftPlan plan_m_, plan_h_;
    // Compile-time FP32 iteration kernels (kernels_ct.cuh): the catalog
    // split of each axis when the axis has one (empty: run-time plans), and
    // its twiddle table.  plan_m_/plan_h_ then hold a run-time split of the
    // same length for the setup and batched kernels.
    std::vector<int> ct_row_rad_, ct_col_rad_;
    cx<T> *ct_tw_row_ = nullptr, *ct_tw_col_ = nullptr;
    bool ct_rows() const { return sizeof(T) == 4 && !ct_row_rad_.empty() && use_tma_ && row_b_ == 2; }
    bool ct_cols() const { return sizeof(T) == 4 && !ct_col_rad_.empty(); }
    cx<T> *post_ = nullptr;
    T *estimate_ = nullptr, *coverage_ = nullptr, *den_ = nullptr, *correction_ = nullptr;
    T *blur_ = nullptr, *wr_ = nullptr, *scatter_ = nullptr, *sci_ = nullptr, *wht_ = nullptr;
    uint8_t *frozen_ = nullptr;
    cx<T> *rx_ = nullptr, *y_ = nullptr, *rs_ = nullptr, *cr_ = nullptr, *khat_ = nullptr;
    cx<T> *aux_fwd_ = nullptr;
    void *aux_adj_ = nullptr;
    ExpDesc<T> *d_exps_ = nullptr;
    ExpStats *d_stats_ = nullptr;
    unsigned long long *d_err_ = nullptr, *d_red_neg_ = nullptr, *d_part_neg_ = nullptr;
    double *d_part_sum_ = nullptr, *d_red_sum_ = nullptr;
    int upd_grid_ = 0;
    unsigned *d_upd_done_ = nullptr;
    T weight_scale_ = 0, max_sens_ = 0;
    uint64_t masked_ = 0;
    void *pinned_ = nullptr;
    size_t pinned_bytes_ = 0;
    std::vector<cudaEvent_t> events_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;

    template <typename U> U *alloc(size_t n) {
        U *p = dalloc<U>(n, &bytes_);
        allocs_.push_back(p);
        return p;
    }
    size_t rec_stride() const { return align16(nexp_ * sizeof(ExpStats) + 24); }
    void ensure_pinned(size_t bytes) {
        if (bytes <= pinned_bytes_) return;
        drop_loop_graphs();  // they copy into the old buffer
        if (pinned_) cudaFreeHost(pinned_);
        UPDC_CUDA(cudaMallocHost(&pinned_, bytes));
        pinned_bytes_ = bytes;
    }

    bool acc_fp64() const { return opt_.form == FORM_FP32 && sizeof(T) == 4; }

    // ------------------------------------------------------------------ FFT shape and autotuner
    // The padded FFT shape follows select_fft_shape (updc_core.c:242-291):
    // without autotuning the smallest 7-smooth sizes >= W + pw - 1 and
    // H + ph - 1 (even width here: the row transform is a half-length complex
    // FFT).  With autotuning the candidate shapes are the reference's (five
    // fast sizes per axis, the diagonal pairs and four off-diagonal ones), and
    // for each axis length every radix split within one stage of the fewest is
    // timed with the engine's own row and column kernels on scratch planes;
    // the shape with the smallest modelled spectral time per iteration wins.
    // The choice is cached like the reference's fft_autotune_v1 files
    // (updc_core.c:195-230), keyed by the device instead of FFTW's version.
    FftChoice choice_;
    const FftChoice &fft_choice() const override { return choice_; }

    static std::vector<int> fast_candidates(int minimum, bool even, int count, int cap) {
        std::vector<int> out;
        for (int v = minimum; (int)out.size() < count; ++v) {
            v = next_smooth(v, even);
            if (v > cap) break;
            out.push_back(v);
        }
        return out;
    }

    std::string tune_cache_path(int min_w, int min_h) const {
        if (opt_.tune_cache_dir.empty()) return "";
        char name[160];
        snprintf(name, sizeof(name), "fft_autotune_b200_v1_%s_%dx%d_h%d_n%d.txt", sizeof(T) == 4 ? "f32" : "f64",
                 min_w, min_h, H_, nexp_);
        return opt_.tune_cache_dir + "/" + name;
    }
    std::string device_signature() const {
        cudaDeviceProp p;
        UPDC_CUDA(cudaGetDeviceProperties(&p, opt_.device));
        int rt = 0;
        cudaRuntimeGetVersion(&rt);
        char sig[400];
        snprintf(sig, sizeof(sig), "%s|sm%d%d|%d SMs|cudart %d|updc_b200 tuner 2", p.name, p.major, p.minor,
                 p.multiProcessorCount, rt);
        return sig;
    }
    static std::string radix_text(const std::vector<int> &r) {
        std::string t;
        for (size_t i = 0; i < r.size(); ++i) t += (i ? "," : "") + std::to_string(r[i]);
        return t;
    }
    static std::vector<int> radix_parse(const char *t) {
        std::vector<int> r;
        for (const char *c = t; *c;) {
            char *e = nullptr;
            const long v = strtol(c, &e, 10);
            if (e == c) break;
            r.push_back((int)v);
            c = *e == ',' ? e + 1 : e;
        }
        return r;
    }
    bool load_tune_cache(const std::string &path, int min_w, int min_h, FftChoice &c) const {
        if (path.empty() || opt_.retune) return false;
        FILE *f = fopen(path.c_str(), "r");
        if (!f) return false;
        char sig[400] = {}, rr[200] = {}, cr[200] = {};
        int mw = 0, mh = 0, w = 0, h = 0;
        double ms = 0;
        const bool ok = fscanf(f, "signature=%399[^\n]\nmin_width=%d\nmin_height=%d\nwidth=%d\nheight=%d\n"
                                  "row_radices=%199[^\n]\ncol_radices=%199[^\n]\npredicted_ms=%lf\n",
                               sig, &mw, &mh, &w, &h, rr, cr, &ms) == 8;
        fclose(f);
        if (!ok || device_signature() != sig || mw != min_w || mh != min_h || w < min_w || h < min_h || (w & 1))
            return false;
        c.width = w;
        c.height = h;
        c.row_radices = radix_parse(rr);
        c.col_radices = radix_parse(cr);
        c.predicted_ms = ms;
        long pr = 1, pc = 1;
        for (int r : c.row_radices) pr *= r;
        for (int r : c.col_radices) pc *= r;
        return pr == w / 2 && pc == h;
    }
    void save_tune_cache(const std::string &path, int min_w, int min_h, const FftChoice &c) const {
        if (path.empty()) return;
        const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
        FILE *f = fopen(tmp.c_str(), "w");
        if (!f) return;
        fprintf(f, "signature=%s\nmin_width=%d\nmin_height=%d\nwidth=%d\nheight=%d\nrow_radices=%s\ncol_radices=%s\n"
                   "predicted_ms=%.6f\n",
                device_signature().c_str(), min_w, min_h, c.width, c.height, radix_text(c.row_radices).c_str(),
                radix_text(c.col_radices).c_str(), c.predicted_ms);
        if (fclose(f) || rename(tmp.c_str(), path.c_str())) unlink(tmp.c_str());
    }

    // Device time (ms, best of 3 after one warm-up) of a launch sequence.
    template <class F> float time_launch(F &&launch) {
        cudaEvent_t a, b;
        UPDC_CUDA(cudaEventCreate(&a));
        UPDC_CUDA(cudaEventCreate(&b));
        float best = 1e30f;
        launch();
        for (int r = 0; r < 3; ++r) {
            UPDC_CUDA(cudaEventRecord(a, stream_));
            launch();
            UPDC_CUDA(cudaEventRecord(b, stream_));
            UPDC_CUDA(cudaEventSynchronize(b));
            float ms = 0;
            UPDC_CUDA(cudaEventElapsedTime(&ms, a, b));
            best = std::min(best, ms);
        }
        UPDC_CUDA(cudaGetLastError());
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return best;
    }

    // Candidate splits of an axis length (at most one stage more than the
    // fewest), fewest stages first, at most 20.
    static std::vector<std::vector<int>> split_candidates(int n) {
        std::vector<std::vector<int>> all;
        fft_factorizations(n, FFT_RMAX, 1, all);
        std::stable_sort(all.begin(), all.end(), [](const std::vector<int> &a, const std::vector<int> &b) {
            return a.size() < b.size();
        });
        if (all.size() > 20) all.resize(20);
        return all;
    }

    // Times the row transform (R2C of H rows of a W-wide plane into an M-point
    // spectrum) for every split of M; returns the best split and its time.
    std::pair<std::vector<int>, float> tune_row(int M, const T *plane, cx<T> *spec, int ld, int *timed) {
        std::pair<std::vector<int>, float> best{{}, 1e30f};
        const int nu = M + 1, fw = 2 * M;
        int B = std::max(1, std::min(Caps<T>::ROW / M, H_));
        if (sizeof(T) == 4 && B >= 2) B &= ~1;
        std::vector<cx<T>> post(nu);
        const double two_pi = 6.283185307179586476925286766559;
        for (int u = 0; u <= M; ++u) post[u] = cx<T>{(T)std::cos(-two_pi * u / fw), (T)std::sin(-two_pi * u / fw)};
        cx<T> *dpost = dalloc<cx<T>>(nu, nullptr);
        UPDC_CUDA(cudaMemcpy(dpost, post.data(), nu * sizeof(cx<T>), cudaMemcpyHostToDevice));
        for (const auto &rad : split_candidates(M)) {
            FftPlan plan;
            auto tab = fft_make_table<T>(M, rad, plan);
            plan.pad_shift = fft_choose_padding(plan, RowNt<T>::value, Caps<T>::ROW, std::max(1, std::min(2, Caps<T>::ROW / M)));
            const size_t smem = row_buf_bytes(B, M, sizeof(cx<T>), plan.pad_shift);
            if (smem > SMEM_LIMIT) continue;
            cx<T> *dtab = dalloc<cx<T>>(tab.size(), nullptr);
            UPDC_CUDA(cudaMemcpy(dtab, tab.data(), tab.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
            plan.tw = dtab;
            const PlaneLoader<T> pl{plane, W_, 0};
            dim3 grid((unsigned)ceil_div(H_, B), 1);
            float ms = 0;
            by_pad(plan.pad_shift, [&](auto P) {
                by_rows(B, [&](auto Q) {
                    constexpr int PS = decltype(P)::value, BR = decltype(Q)::value;
                    set_smem(k_row_r2c<T, RowNt<T>::value, Caps<T>::ROW, PlaneLoader<T>, false, PS, BR>, smem);
                    ms = time_launch([&] {
                        k_row_r2c<T, RowNt<T>::value, Caps<T>::ROW, PlaneLoader<T>, false, PS, BR>
                            <<<grid, RowNt<T>::value, smem, stream_>>>(plan, dpost, pl, W_, H_, B, FastDiv((uint32_t)B),
                                                                       SpecRef{spec, ld, 0}, no_map_);
                    });
                });
            });
            ++*timed;
            cudaFree(dtab);
            if (ms < best.second) best = {rad, ms};
        }
        // the compile-time kernels of the catalog splits of M (FP32; two-row
        // TMA tiles, as the iteration runs them)
        if constexpr (sizeof(T) == 4) {
            if (B == 2 && ld % 2 == 0)
                for (const auto &rad : ct_catalog_splits(0, M)) {
                    FftPlan unused;
                    auto tab = fft_make_table<T>(M, rad, unused);
                    cx<T> *dtab = dalloc<cx<T>>(tab.size(), nullptr);
                    UPDC_CUDA(cudaMemcpy(dtab, tab.data(), tab.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
                    CUtensorMap map;
                    make_tensor_map_3d(&map, spec, (uint64_t)ld, (uint64_t)M + 1, 1, 2, (uint32_t)row_ubox(M));
                    const size_t smem = row_tma_smem(2, M, sizeof(cx<float>), 31);
                    float ms = 1e30f;
                    ct_row_catalog(rad, [&](auto L) {
                        tune_row_ct(L, smem);
                        ms = time_launch([&] { launch_tune_row_ct(L, dpost, plane, dtab, map, smem); });
                    });
                    ++*timed;
                    cudaFree(dtab);
                    if (ms < best.second) best = {rad, ms};
                }
        }
        cudaFree(dpost);
        return best;
    }
    template <int... R> void tune_row_ct(CtRadices<R...>, size_t smem) { set_smem(k_row_r2c_ct<CT_ROW_NT, 2, R...>, smem); }
    template <int... R>
    void launch_tune_row_ct(CtRadices<R...>, const cx<T> *post, const T *plane, const cx<T> *tw, const CUtensorMap &map,
                            size_t smem) {
        dim3 grid((unsigned)ceil_div(H_, 2), 1);
        k_row_r2c_ct<CT_ROW_NT, 2, R...><<<grid, CT_ROW_NT, smem, stream_>>>(reinterpret_cast<const cx<float> *>(post),
                                                                 reinterpret_cast<const float *>(plane), W_, H_, 0,
                                                                 reinterpret_cast<const cx<float> *>(tw), map);
    }

    // Times the column transform (nc columns of length FH, H input rows) for
    // every split of FH; returns the best split and its time per column.
    std::pair<std::vector<int>, float> tune_col(int FH, int nc, const cx<T> *in, int ld, cx<T> *out, int *timed) {
        std::pair<std::vector<int>, float> best{{}, 1e30f};
        for (const auto &rad : split_candidates(FH)) {
            FftPlan plan;
            auto tab = fft_make_table<T>(FH, rad, plan);
            plan.pad_shift = fft_choose_padding(plan, ColNt<T>::value, Caps<T>::COL_S, 1);
            const size_t smem = fft_buf_bytes(FH, sizeof(cx<T>), plan.pad_shift);
            if (smem > SMEM_LIMIT) continue;
            cx<T> *dtab = dalloc<cx<T>>(tab.size(), nullptr);
            UPDC_CUDA(cudaMemcpy(dtab, tab.data(), tab.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
            plan.tw = dtab;
            float ms = 0;
            constexpr int CNT = ColNt<T>::value;
            by_pad(plan.pad_shift, [&](auto P) {
                constexpr int PS = decltype(P)::value;
                if (FH <= Caps<T>::COL_S) {
                    set_smem(k_col_fft<T, CNT, Caps<T>::COL_S, false, PS>, smem);
                    ms = time_launch([&] {
                        k_col_fft<T, CNT, Caps<T>::COL_S, false, PS><<<(unsigned)nc, CNT, smem, stream_>>>(plan, in, ld, H_, out, FH, FH);
                    });
                } else {
                    set_smem(k_col_fft<T, CNT, Caps<T>::COL_L, false, PS>, smem);
                    ms = time_launch([&] {
                        k_col_fft<T, CNT, Caps<T>::COL_L, false, PS><<<(unsigned)nc, CNT, smem, stream_>>>(plan, in, ld, H_, out, FH, FH);
                    });
                }
            });
            ++*timed;
            cudaFree(dtab);
            if (ms / nc < best.second) best = {rad, ms / nc};
        }
        // the compile-time column kernels of the catalog splits of FH (FP32):
        // the forward column kernel with no exposures is one transform
        if constexpr (sizeof(T) == 4) {
            for (const auto &rad : ct_catalog_splits(1, FH)) {
                FftPlan unused;
                auto tab = fft_make_table<T>(FH, rad, unused);
                cx<T> *dtab = dalloc<cx<T>>(tab.size(), nullptr);
                UPDC_CUDA(cudaMemcpy(dtab, tab.data(), tab.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
                float ms = 1e30f;
                ct_col_catalog(rad, [&](auto L) {
                    ms = time_launch([&] { launch_tune_col_ct(L, nc, in, ld, out, dtab); });
                });
                ++*timed;
                cudaFree(dtab);
                if (ms / nc < best.second) best = {rad, ms / nc};
            }
        }
        return best;
    }
    template <int... R>
    void launch_tune_col_ct(CtRadices<R...>, int nc, const cx<T> *in, int ld, cx<T> *out, const cx<T> *tw) {
        const size_t b = (size_t)CtProd<R...>::value * sizeof(cx<float>);
        set_smem(k_col_forward_ct<CT_COL_NT, R...>, b);
        k_col_forward_ct<CT_COL_NT, R...><<<(unsigned)nc, CT_COL_NT, b, stream_>>>(
            reinterpret_cast<const cx<float> *>(in), ld, H_, nullptr, 0, 0, nullptr, 0, 0, 0,
            reinterpret_cast<cx<float> *>(out), reinterpret_cast<const cx<float> *>(tw));
    }

    void autotune_shape(int min_w, int min_h, FftChoice &c) {
        const double t0 = now_s();
        std::vector<int> wc = opt_.fft_width ? std::vector<int>{opt_.fft_width}
                                             : fast_candidates(min_w, true, 5, 2 * Caps<T>::ROW);
        std::vector<int> hc = opt_.fft_height ? std::vector<int>{opt_.fft_height}
                                              : fast_candidates(min_h, false, 5, Caps<T>::COL_L);
        if (wc.empty() || hc.empty()) throw Error(1, "no FFT shape within the transform capacity");
        std::vector<std::pair<int, int>> shapes;
        auto add = [&](size_t i, size_t j) {
            if (i >= wc.size() || j >= hc.size()) return;
            for (auto &s : shapes)
                if (s.first == wc[i] && s.second == hc[j]) return;
            shapes.push_back({wc[i], hc[j]});
        };
        for (size_t i = 0; i < std::min(wc.size(), hc.size()); ++i) add(i, i);
        add(2, 0), add(0, 2), add(4, 0), add(0, 4);
        if (wc.size() == 1 || hc.size() == 1)
            for (size_t i = 0; i < wc.size(); ++i)
                for (size_t j = 0; j < hc.size(); ++j) add(i, j);
        // scratch: one target plane, its widest row spectrum, NC columns out
        const int NC = 148 * 8;
        const int mmax = *std::max_element(wc.begin(), wc.end()) / 2;
        const int hmax = *std::max_element(hc.begin(), hc.end());
        T *plane = dalloc<T>(nout_, nullptr);
        UPDC_CUDA(cudaMemset(plane, 0, nout_ * sizeof(T)));
        // spectra at the iteration's pitch (even for FP32: TMA strides)
        const int ld = sizeof(T) == 4 ? (H_ + 1) & ~1 : H_;
        cx<T> *spec = dalloc<cx<T>>((size_t)(mmax + 1) * ld, nullptr);
        cx<T> *cols = dalloc<cx<T>>((size_t)NC * hmax, nullptr);
        UPDC_CUDA(cudaMemset(spec, 0, (size_t)(mmax + 1) * ld * sizeof(cx<T>)));
        std::map<int, std::pair<std::vector<int>, float>> rows, colsb;
        int timed = 0;
        try {
            for (auto &s : shapes) {
                if (!rows.count(s.first / 2)) rows[s.first / 2] = tune_row(s.first / 2, plane, spec, ld, &timed);
                if (!colsb.count(s.second))
                    colsb[s.second] = tune_col(s.second, std::min(NC, mmax + 1), spec, ld, cols, &timed);
            }
        } catch (...) {
            cudaFree(plane), cudaFree(spec), cudaFree(cols);
            throw;
        }
        cudaFree(plane), cudaFree(spec), cudaFree(cols);
        // per iteration: 2N+2 row passes and 2N+2 column transforms over
        // M+1 columns, plus 2N reads of a PSF spectrum (HBM, ~6.5 TB/s)
        double best = 1e300;
        for (auto &s : shapes) {
            const auto &r = rows[s.first / 2], &q = colsb[s.second];
            if (r.first.empty() || q.first.empty()) continue;
            const int nu = s.first / 2 + 1;
            const double otf_ms = 2.0 * nexp_ * (double)nu * s.second * sizeof(cx<T>) / 6.5e12 * 1e3;
            const double ms = (2.0 * nexp_ + 2.0) * (r.second + (double)q.second * nu) + otf_ms;
            if (opt_.verbose)
                printf("FFT candidate %dx%d rows [%s] %.4f ms, columns [%s] %.4f ms, modelled %.3f ms/iteration\n",
                       s.first, s.second, radix_text(r.first).c_str(), r.second, radix_text(q.first).c_str(),
                       q.second * nu, ms);
            if (ms < best) {
                best = ms;
                c.width = s.first;
                c.height = s.second;
                c.row_radices = r.first;
                c.col_radices = q.first;
            }
        }
        if (c.row_radices.empty()) throw Error(1, "FFT autotune found no usable plan");
        c.predicted_ms = best;
        c.candidates = timed;
        c.seconds = now_s() - t0;
    }

    // Smallest circular length of one axis for a grid of n pixels and PSFs
    // of extent f along it.  PSF pixel x sits at circular offset x - f/2
    // (updc_core.c:814-819), in [-(f/2), f - 1 - f/2].  The forward model
    // keeps outputs y < n of sum_t x[(y - t) mod F] psf[t] and the adjoint of
    // sum_t s[(y + t) mod F] psf[t]; with x and s zero beyond n, every index
    // that wraps lands in the zero padding exactly when F >= n + f/2, and
    // the PSF does not overlap itself when F >= f.  At that length the kept
    // window equals the linear convolution's, which the reference computes
    // with F >= n + f - 1 (updc_core.c:1335-1341); fft_linear keeps that rule.
    int min_fft_length(int n, int f) const {
        if (opt_.fft_linear) return n + f - 1;
        return std::max(n + f / 2, f);
    }

    void choose_fft_shape() {
        int mpw = 0, mph = 0;
        for (auto &e : exps_) {
            mpw = std::max(mpw, e.psf_width);
            mph = std::max(mph, e.psf_height);
        }
        const int pad_w = transposed_ ? mph : mpw, pad_h = transposed_ ? mpw : mph;
        const int min_w = min_fft_length(W_, pad_w), min_h = min_fft_length(H_, pad_h);
        if ((opt_.fft_width && (opt_.fft_width < min_w || (opt_.fft_width & 1))) || (opt_.fft_height && opt_.fft_height < min_h))
            throw Error(1, "FFT shape below the minimum length or odd width");
        FftChoice c;
        // rows longer than one block holds (FW/2 above the row capacity) take
        // the four-step long-row kernels at the smallest width; the
        // autotuner times single-block row splits only
        const bool long_min = min_w / 2 > Caps<T>::ROW || (opt_.fft_width && opt_.fft_width / 2 > Caps<T>::ROW) ||
                              min_h > Caps<T>::COL_L || opt_.fft_height > Caps<T>::COL_L;
        if (opt_.autotune && !long_min) {
            const std::string cache = tune_cache_path(min_w, min_h);
            const double t0 = now_s();
            if (load_tune_cache(cache, min_w, min_h, c) && (!opt_.fft_width || c.width == opt_.fft_width) &&
                (!opt_.fft_height || c.height == opt_.fft_height)) {
                c.cache_hit = true;
                c.seconds = now_s() - t0;
            } else {
                c = FftChoice();
                autotune_shape(min_w, min_h, c);
                save_tune_cache(cache, min_w, min_h, c);
            }
        } else {
            c.width = opt_.fft_width ? opt_.fft_width : next_smooth(min_w, true);
            c.height = opt_.fft_height ? opt_.fft_height : next_smooth(min_h, false);
        }
        FW_ = c.width;
        FH_ = c.height;
        M_ = FW_ / 2;
        long_rows_ = M_ > Caps<T>::ROW;
        if (long_rows_ && !long_row_split(M_, Caps<T>::ROW, lrp_.M1, lrp_.M2))
            throw Error(1, "FFT width exceeds the row-transform capacity");
        long_cols_ = FH_ > Caps<T>::COL_L;
        if (long_cols_ && !long_col_split(FH_, Caps<T>::COL_L, lcp_.N1, lcp_.N2))
            throw Error(1, "FFT height exceeds the column-transform capacity");
        // a catalog split (compile-time kernels) is preferred where the length
        // has one and nothing was tuned; a split that is neither a catalog
        // entry nor a valid run-time one (non-increasing radices <= 16, e.g.
        // from another build's cache) is replaced by the greedy split
        ct_row_rad_.clear();
        ct_col_rad_.clear();
        if (sizeof(T) == 4) {
            if (c.row_radices.empty()) {
                const auto cs = ct_catalog_splits(0, M_);
                if (!cs.empty()) c.row_radices = cs[0];
            }
            if (c.col_radices.empty()) {
                const auto cs = ct_catalog_splits(1, FH_);
                if (!cs.empty()) c.col_radices = cs[0];
            }
            if (ct_row_catalog(c.row_radices, [](auto) {})) ct_row_rad_ = c.row_radices;
            if (ct_col_catalog(c.col_radices, [](auto) {})) ct_col_rad_ = c.col_radices;
        }
        auto runtime_split = [](int n, const std::vector<int> &rad) {
            long p = 1;
            for (size_t i = 0; i < rad.size(); ++i) {
                if (rad[i] > FFT_RMAX || (i && rad[i] > rad[i - 1])) return false;
                p *= rad[i];
            }
            return !rad.empty() && p == n;
        };
        std::vector<int> gen_row = c.row_radices, gen_col = c.col_radices;
        if (!runtime_split(M_, gen_row) && !fft_factor(M_, FFT_RMAX, gen_row))
            throw Error(1, "FFT length " + std::to_string(M_) + " is not 7-smooth");
        if (!runtime_split(FH_, gen_col) && !fft_factor(FH_, FFT_RMAX, gen_col))
            throw Error(1, "FFT length " + std::to_string(FH_) + " is not 7-smooth");
        if (ct_row_rad_.empty()) c.row_radices = gen_row;
        if (ct_col_rad_.empty()) c.col_radices = gen_col;
        choice_ = c;
        // twiddle tables
        auto tm = fft_make_table<T>(M_, gen_row, plan_m_);
        auto th = fft_make_table<T>(FH_, gen_col, plan_h_);
        for (int axis = 0; axis < 2; ++axis) {
            const std::vector<int> &rad = axis ? ct_col_rad_ : ct_row_rad_;
            if (rad.empty()) continue;
            FftPlan unused;
            auto t = fft_make_table<T>(axis ? FH_ : M_, rad, unused);
            cx<T> *d = alloc<cx<T>>(t.size());
            UPDC_CUDA(cudaMemcpy(d, t.data(), t.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
            (axis ? ct_tw_col_ : ct_tw_row_) = d;
        }
        plan_m_.pad_shift = fft_choose_padding(plan_m_, RowNt<T>::value, Caps<T>::ROW, std::max(1, std::min(2, Caps<T>::ROW / M_)));
        plan_h_.pad_shift = long_cols_ ? 31 : fft_choose_padding(plan_h_, ColNt<T>::value, Caps<T>::COL_S, 1);
        cx<T> *dm = alloc<cx<T>>(tm.size()), *dh = alloc<cx<T>>(th.size());
        UPDC_CUDA(cudaMemcpy(dm, tm.data(), tm.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
        UPDC_CUDA(cudaMemcpy(dh, th.data(), th.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
        plan_m_.tw = dm;
        plan_h_.tw = dh;
        std::vector<cx<T>> post(M_ + 1);
        const double two_pi = 6.283185307179586476925286766559;
        for (int u = 0; u <= M_; ++u) post[u] = cx<T>{(T)std::cos(-two_pi * u / FW_), (T)std::sin(-two_pi * u / FW_)};
        post_ = alloc<cx<T>>(M_ + 1);
        UPDC_CUDA(cudaMemcpy(post_, post.data(), post.size() * sizeof(cx<T>), cudaMemcpyHostToDevice));
        if (long_rows_) lrp_ = make_long_plan<T>(lrp_.M1, lrp_.M2, [&](size_t n) { return (void *)alloc<cx<T>>(n); });
        if (long_cols_) lcp_ = col_plan(make_long_plan<T>(lcp_.N1, lcp_.N2, [&](size_t n) { return (void *)alloc<cx<T>>(n); }));
    }

    // ------------------------------------------------------------------ long columns (longrow.cuh)
    bool long_cols_ = false;
    LongColPlan lcp_;
    cx<T> *long_col_scratch_ = nullptr, *long_col_tmp_ = nullptr;  // (M+1) x FH each
    static LongColPlan col_plan(const LongRowPlan &r) {
        LongColPlan c;
        c.N = r.M, c.N1 = r.M1, c.N2 = r.M2, c.p1 = r.p1, c.p2 = r.p2, c.twm = r.twm;
        return c;
    }
    // Column FFTs (forward, or unnormalised inverse) of length FH of `ncols`
    // u-rows, four-step: rows [0, rows_in) of each input column (zero beyond)
    // to rows [0, rows_out) of the output.
    template <typename U, bool INV>
    void long_col_fft(const LongColPlan &lp, const cx<U> *in, int ld_in, int rows_in, cx<U> *out, int ld_out,
                      int rows_out, int ncols, cx<U> *scratch) {
        constexpr int CAP = Caps<U>::COL_L;
        const size_t sa = (size_t)LONG_G * lp.N2 * sizeof(cx<U>), sb = (size_t)LONG_G * lp.N1 * sizeof(cx<U>);
        set_smem(k_long_col_a<U, NT, CAP, INV>, sa);
        set_smem(k_long_col_b<U, NT, CAP, INV>, sb);
        k_long_col_a<U, NT, CAP, INV><<<dim3((unsigned)ceil_div(lp.N1, LONG_G), ncols), NT, sa, stream_>>>(
            lp, in, ld_in, rows_in, scratch);
        k_long_col_b<U, NT, CAP, INV><<<dim3((unsigned)ceil_div(lp.N2, LONG_G), ncols), NT, sb, stream_>>>(
            lp, scratch, out, ld_out, rows_out);
        UPDC_CUDA(cudaGetLastError());
    }
    void configure_long_cols() {
        const size_t sa = (size_t)LONG_G * lcp_.N2 * sizeof(cx<T>), sb = (size_t)LONG_G * lcp_.N1 * sizeof(cx<T>);
        constexpr int CAP = Caps<T>::COL_L;
        set_smem(k_long_col_a<T, NT, CAP, false>, sa);
        set_smem(k_long_col_a<T, NT, CAP, true>, sa);
        set_smem(k_long_col_b<T, NT, CAP, false>, sb);
        set_smem(k_long_col_b<T, NT, CAP, true>, sb);
    }
    // Forward model, columns: X-hat = FFT(pad(rx)), then IFFT(X-hat K_k) per
    // active exposure into its y spectrum (unnormalised, rows < H).
    void long_col_forward() {
        const size_t nu = (size_t)M_ + 1, n = nu * FH_;
        cx<T> *xh = aux_fwd_;
        long_col_fft<T, false>(lcp_, rx_, ldh_, H_, xh, FH_, FH_, (int)nu, long_col_scratch_);
        for (int j = 0; j < act_n_; ++j) {
            const int k = act_k0_ + j;
            k_long_mul<T><<<grid1d(n), 256, 0, stream_>>>(xh, khat_ + (size_t)k * n, long_col_tmp_, n);
            long_col_fft<T, true>(lcp_, long_col_tmp_, FH_, FH_, y_ + (size_t)k * nu * ldh_, ldh_, H_, (int)nu,
                                  long_col_scratch_);
        }
        UPDC_CUDA(cudaGetLastError());
    }
    // Adjoint, columns: the conj-OTF products of the active exposures' scatter
    // spectra summed through the form's accumulator, then the inverse into cr.
    template <class Acc> void long_col_adjoint(const cx<T> *khat) {
        const size_t nu = (size_t)M_ + 1, n = nu * FH_;
        auto *acc = (typename Acc::S *)aux_adj_;
        for (int j = 0; j < act_n_; ++j) {
            const int k = act_k0_ + j;
            long_col_fft<T, false>(lcp_, rs_ + (size_t)k * nu * ldh_, ldh_, H_, long_col_tmp_, FH_, FH_, (int)nu,
                                   long_col_scratch_);
            k_long_acc<T, Acc><<<grid1d(n), 256, 0, stream_>>>(long_col_tmp_, khat + (size_t)k * n, acc, n, j == 0);
        }
        k_long_get<T, Acc><<<grid1d(n), 256, 0, stream_>>>(acc, long_col_tmp_, n);
        long_col_fft<T, true>(lcp_, long_col_tmp_, FH_, FH_, cr_, ldh_, H_, (int)nu, long_col_scratch_);
    }

    // ------------------------------------------------------------------ long rows (longrow.cuh)
    bool long_rows_ = false;
    LongRowPlan lrp_;
    cx<T> *long_scratch_ = nullptr;  // planes x rows x M of the long-row passes
    // Plans and tables of precision U for M = M1 * M2; `get(n)` allocates n
    // complex values of U on the device.
    template <typename U, class Get> LongRowPlan make_long_plan(int M1, int M2, Get &&get) {
        LongRowPlan lp;
        lp.M1 = M1, lp.M2 = M2, lp.M = M1 * M2;
        auto t1 = fft_make_table<U>(M1, FFT_RMAX, lp.p1);
        auto t2 = fft_make_table<U>(M2, FFT_RMAX, lp.p2);
        lp.p1.pad_shift = lp.p2.pad_shift = 31;
        std::vector<cx<U>> tm(lp.M);
        const double two_pi = 6.283185307179586476925286766559;
        for (int e = 0; e < lp.M; ++e) tm[e] = cx<U>{(U)std::cos(-two_pi * e / lp.M), (U)std::sin(-two_pi * e / lp.M)};
        cx<U> *d1 = (cx<U> *)get(t1.size()), *d2 = (cx<U> *)get(t2.size()), *dm = (cx<U> *)get(tm.size());
        UPDC_CUDA(cudaMemcpy(d1, t1.data(), t1.size() * sizeof(cx<U>), cudaMemcpyHostToDevice));
        UPDC_CUDA(cudaMemcpy(d2, t2.data(), t2.size() * sizeof(cx<U>), cudaMemcpyHostToDevice));
        UPDC_CUDA(cudaMemcpy(dm, tm.data(), tm.size() * sizeof(cx<U>), cudaMemcpyHostToDevice));
        lp.p1.tw = d1;
        lp.p2.tw = d2;
        lp.twm = dm;
        return lp;
    }
    // Real rows [0, rows) of `planes` planes (through the loader) -> u-major
    // bins in `out`, four-step; `scratch` holds planes x rows x M.
    template <typename U, class Loader>
    void long_r2c(const LongRowPlan &lp, const Loader &ld, int W, int rows, int planes, const cx<U> *post, SpecRef out,
                  cx<U> *scratch) {
        constexpr int NT = RowNt<U>::value, CAP = Caps<U>::ROW;
        const size_t sa = (size_t)LONG_G * lp.M2 * sizeof(cx<U>), sb = 2 * (size_t)lp.M1 * sizeof(cx<U>);
        set_smem(k_long_r2c_a<U, NT, CAP, Loader>, sa);
        set_smem(k_long_r2c_b<U, NT, CAP>, sb);
        k_long_r2c_a<U, NT, CAP, Loader><<<dim3((unsigned)ceil_div(lp.M1, LONG_G), rows, planes), NT, sa, stream_>>>(
            lp, ld, W, rows, scratch);
        k_long_r2c_b<U, NT, CAP><<<dim3((unsigned)(lp.M2 / 2 + 1), rows, planes), NT, sb, stream_>>>(lp, scratch, post,
                                                                                                   rows, out);
        UPDC_CUDA(cudaGetLastError());
    }
    // u-major bins `in` of `planes` planes -> cropped, scaled real rows through
    // the epilogue, four-step.
    template <typename U, class Epi>
    void long_c2r(const LongRowPlan &lp, const cx<U> *post, SpecRef in, int rows, int planes, int W, U scale,
                  const Epi &epi, cx<U> *scratch) {
        constexpr int NT = RowNt<U>::value, CAP = Caps<U>::ROW;
        const size_t sa = 2 * (size_t)lp.M1 * sizeof(cx<U>), sb = (size_t)LONG_G * lp.M2 * sizeof(cx<U>);
        set_smem(k_long_c2r_a<U, NT, CAP>, sa);
        set_smem(k_long_c2r_b<U, NT, CAP, Epi>, sb);
        k_long_c2r_a<U, NT, CAP><<<dim3((unsigned)ceil_div(lp.M2, 2), rows, planes), NT, sa, stream_>>>(lp, post, in, rows,
                                                                                                      scratch);
        k_long_c2r_b<U, NT, CAP, Epi><<<dim3((unsigned)ceil_div(lp.M1, LONG_G), rows, planes), NT, sb, stream_>>>(
            lp, scratch, rows, W, scale, epi);
        UPDC_CUDA(cudaGetLastError());
    }

    void allocate() {
        const size_t nu = (size_t)M_ + 1;
        // u-major spectra keep H rows at an even pitch for FP32 so that every
        // u-row starts on a 16-byte boundary (TMA strides are multiples of 16)
        ldh_ = sizeof(T) == 4 ? (H_ + 1) & ~1 : H_;
        estimate_ = alloc<T>(nout_);
        coverage_ = alloc<T>(nout_);
        den_ = alloc<T>(nout_);
        correction_ = alloc<T>(nout_);
        blur_ = alloc<T>(nexp_ * nout_);
        scatter_ = alloc<T>(nexp_ * nout_);
        wr_ = alloc<T>(nexp_ * nin_);
        sci_ = alloc<T>(nexp_ * nin_);
        wht_ = alloc<T>(nexp_ * nin_);
        frozen_ = alloc<uint8_t>(nexp_ * nin_);
        UPDC_CUDA(cudaMemset(frozen_, 0, nexp_ * nin_));
        rx_ = alloc<cx<T>>(nu * ldh_);
        cr_ = alloc<cx<T>>(nu * ldh_);
        y_ = alloc<cx<T>>(nexp_ * nu * ldh_);
        rs_ = alloc<cx<T>>(nexp_ * nu * ldh_);
        for (auto *p : {rx_, cr_}) UPDC_CUDA(cudaMemset(p, 0, nu * ldh_ * sizeof(cx<T>)));
        for (auto *p : {y_, rs_}) UPDC_CUDA(cudaMemset(p, 0, nexp_ * nu * ldh_ * sizeof(cx<T>)));
        khat_ = alloc<cx<T>>(nexp_ * nu * FH_);
        d_exps_ = alloc<ExpDesc<T>>(nexp_);
        d_stats_ = alloc<ExpStats>(nexp_);
        init_stats_template();
        d_err_ = alloc<unsigned long long>(1);
        // 16-byte accesses (Vec16<T>::n pixels per thread and step), at most
        // eight 256-thread blocks per SM
        upd_grid_ = (int)std::max<size_t>(1, std::min<size_t>(ceil_div(nout_ / Vec16<T>::n, 256), 148 * 8));
        d_upd_done_ = alloc<unsigned>(1);
        UPDC_CUDA(cudaMemset(d_upd_done_, 0, sizeof(unsigned)));
        d_part_sum_ = alloc<double>(upd_grid_);
        d_part_neg_ = alloc<unsigned long long>(upd_grid_);
        d_red_sum_ = alloc<double>(1);
        d_red_neg_ = alloc<unsigned long long>(1);
        if (long_cols_ || cols_in_global() ||
            fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift) + align16((size_t)FH_ * sizeof(cx<T>)) > SMEM_LIMIT)
            aux_fwd_ = alloc<cx<T>>(nu * FH_);
        if (long_cols_) {
            long_col_scratch_ = alloc<cx<T>>(nu * FH_);
            long_col_tmp_ = alloc<cx<T>>(nu * FH_);
        }
        links_.assign(nexp_, DevLinkMap());
        // rows per row-transform block; the TMA path needs an even number of
        // 8-byte elements per row tile (16-byte box rows and coordinates)
        constexpr int EW = TmaElems<T>::value;
        row_b_ = std::max(1, std::min({Caps<T>::ROW / M_, TMA_UBOX / EW, ldh_}));
        if (EW == 1 && row_b_ >= 2) row_b_ &= ~1;
        // the FFT buffer and the staging tile share the block's shared memory
        while (row_b_ > 2 && row_tma_smem(row_b_, M_, sizeof(cx<T>), plan_m_.pad_shift) > SMEM_LIMIT)
            row_b_ -= EW == 1 ? 2 : 1;
        // FP32 rows of more than half the capacity: two-row TMA tiles in the
        // 1024-thread "wide" instantiation (one block per SM) instead of
        // one-row tiles with strided 8-byte accesses
        wide_rows_ = sizeof(T) == 4 && !long_rows_ && row_b_ == 1 && M_ > Caps<T>::ROW / 2 && ldh_ >= 2 &&
                     row_tma_smem(2, M_, sizeof(cx<T>), plan_m_.pad_shift) <= SMEM_LIMIT;
        if (wide_rows_) row_b_ = 2;
        use_tma_ = !long_rows_ && (row_b_ * EW) % 2 == 0 &&
                   row_tma_smem(row_b_, M_, sizeof(cx<T>), plan_m_.pad_shift) <= SMEM_LIMIT;
        if (long_rows_) long_scratch_ = alloc<cx<T>>((size_t)std::max(nexp_ * H_, FH_) * M_);
        if (!ct_row_rad_.empty() && !(use_tma_ && row_b_ == 2)) {
            // the compile-time row kernels take two-row TMA tiles
            ct_row_rad_.clear();
            choice_.row_radices.assign(plan_m_.radix, plan_m_.radix + plan_m_.nstage);
        }
        if (use_tma_) {
            const uint64_t d0 = (uint64_t)ldh_ * EW;
            const uint32_t ub = (uint32_t)row_ubox(M_);
            make_tensor_map_3d(&map_rx_, rx_, d0, nu, 1, row_b_ * EW, ub);
            make_tensor_map_3d(&map_cr_, cr_, d0, nu, 1, row_b_ * EW, ub);
        }
        if (!shard_setup_) {
            act_k0_ = 0;
            act_n_ = nexp_;
        }
        build_exposure_maps();
        configure_kernels();
        // the adjoint's accumulator plane, when it does not fit shared memory,
        // is allocated here: iterations are captured into graphs, where no
        // allocation may happen
        if constexpr (sizeof(T) == 4) {
            if (opt_.form == FORM_FP32) ensure_adj_aux<AccF64>();
            else if (opt_.form == FORM_FP32_KAHAN) ensure_adj_aux<AccKahan>();
            else ensure_adj_aux<AccPlain<T>>();
        } else {
            ensure_adj_aux<AccPlain<T>>();
        }
    }

    // ------------------------------------------------------------------ kernel configuration
    int ldh_ = 0, row_b_ = 1;
    bool wide_rows_ = false;
    static constexpr int WIDE_NT = 1024, WIDE_CAP = 2 * Caps<T>::ROW;
    bool use_tma_ = false;
    CUtensorMap map_rx_{}, map_cr_{}, map_y_{}, map_rs_{}, no_map_{};

    size_t row_smem() const {
        return use_tma_ ? row_tma_smem(row_b_, M_, sizeof(cx<T>), plan_m_.pad_shift)
                        : row_buf_bytes(row_b_, M_, sizeof(cx<T>), plan_m_.pad_shift);
    }
    int row_batch() const { return row_b_; }
    size_t fwd_smem() const {
        return fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift) + (aux_fwd_ ? 0 : align16(FH_ * sizeof(cx<T>)));
    }
    // FP32 column kernels keep X-hat and the adjoint accumulator of their
    // column in a global scratch (L2-resident: ~50 MB for all resident
    // blocks) so that three blocks fit an SM.
    static constexpr bool cols_in_global() { return sizeof(T) == 4; }
    template <class Acc> size_t adj_smem() const {
        const size_t b = fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift) + align16(FH_ * sizeof(typename Acc::S));
        return adj_aux<Acc>() ? fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift) : b;
    }
    template <class Acc> bool adj_aux() const {
        return cols_in_global() ||
               fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift) + align16(FH_ * sizeof(typename Acc::S)) > SMEM_LIMIT;
    }

    void configure_kernels() {
        if (long_rows_) {
            // the iteration's long-row launches (attributes set before any capture)
            constexpr int NT = RowNt<T>::value, CAP = Caps<T>::ROW;
            const size_t sg = (size_t)LONG_G * lrp_.M2 * sizeof(cx<T>), s2 = 2 * (size_t)lrp_.M1 * sizeof(cx<T>);
            set_smem(k_long_r2c_a<T, NT, CAP, PlaneLoader<T>>, sg);
            set_smem(k_long_r2c_b<T, NT, CAP>, s2);
            set_smem(k_long_c2r_a<T, NT, CAP>, s2);
            set_smem(k_long_c2r_b<T, NT, CAP, PlaneStore<T>>, sg);
        } else {
            const size_t rs = row_smem();
            if (wide_rows_)
                by_pad(plan_m_.pad_shift, [&](auto P) {
                    constexpr int PS = decltype(P)::value;
                    set_smem(k_row_r2c<T, WIDE_NT, WIDE_CAP, PlaneLoader<T>, true, PS, 2>, rs);
                    set_smem(k_row_c2r<T, WIDE_NT, WIDE_CAP, PlaneStore<T>, true, PS, 2>, rs);
                });
            else by_pad(plan_m_.pad_shift, [&](auto P) {
                by_rows(row_b_, [&](auto Q) {
                    constexpr int PS = decltype(P)::value, BR = decltype(Q)::value;
                    set_smem(k_row_r2c<T, RowNt<T>::value, Caps<T>::ROW, PlaneLoader<T>, true, PS, BR>, rs);
                    set_smem(k_row_r2c<T, RowNt<T>::value, Caps<T>::ROW, PlaneLoader<T>, false, PS, BR>, rs);
                    set_smem(k_row_c2r<T, RowNt<T>::value, Caps<T>::ROW, PlaneStore<T>, true, PS, BR>, rs);
                    set_smem(k_row_c2r<T, RowNt<T>::value, Caps<T>::ROW, PlaneStore<T>, false, PS, BR>, rs);
                });
            });
        }
        set_smem(k_detector<T, true>, sizeof(DetShared));
        set_smem(k_detector<T, false>, sizeof(DetShared));
        if (long_cols_) {
            configure_long_cols();
        } else {
            const size_t fs = fwd_smem();
            by_pad(plan_h_.pad_shift, [&](auto P) {
                constexpr int PS = decltype(P)::value;
                set_smem(k_col_forward<T, ColNt<T>::value, Caps<T>::COL_S, ColAux<T>, PS>, fs);
                set_smem(k_col_forward<T, ColNt<T>::value, Caps<T>::COL_L, ColAux<T>, PS>, fs);
            });
            set_smem(k_col_fft<T, NT, Caps<T>::COL_S, false>, fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift));
            set_smem(k_col_fft<T, NT, Caps<T>::COL_L, false>, fft_buf_bytes(FH_, sizeof(cx<T>), plan_h_.pad_shift));
            configure_adjoint<AccPlain<T>>();
            if (sizeof(T) == 4) {
                configure_adjoint<AccF64>();
                configure_adjoint<AccKahan>();
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (ct_rows())
                ct_row_catalog(ct_row_rad_, [&](auto L) {
                    configure_rows_ct(L);
                });
            if (ct_cols())
                ct_col_catalog(ct_col_rad_, [&](auto L) {
                    configure_cols_ct(L);
                });
        }
    }
    size_t ct_row_smem() const { return row_tma_smem(2, M_, sizeof(cx<float>), 31); }
    template <int... R> void configure_rows_ct(CtRadices<R...>) {
        set_smem(k_gather_row_r2c_ct<CT_ROW_NT, R...>, ct_row_smem());
        set_smem(k_row_r2c_ct<CT_ROW_NT, 2, R...>, ct_row_smem());
        set_smem(k_row_c2r_ct<CT_ROW_NT, 2, R...>, ct_row_smem());
    }
    template <int... R> void configure_cols_ct(CtRadices<R...>) {
        const size_t b = (size_t)FH_ * sizeof(cx<float>);
        set_smem(k_col_forward_ct<CT_COL_NT, R...>, b);
        set_smem(k_col_adjoint_ct<AccF64, CT_COL_NT, R...>, b);
        set_smem(k_col_adjoint_ct<AccKahan, CT_COL_NT, R...>, b);
        set_smem(k_col_adjoint_ct<AccPlain<float>, CT_COL_NT, R...>, b);
    }
    template <int... R>
    void launch_row_r2c_ct(CtRadices<R...>, const float *plane, int batch, size_t plane_stride, const CUtensorMap &map) {
        dim3 grid((unsigned)ceil_div(H_, 2), (unsigned)batch);
        k_row_r2c_ct<CT_ROW_NT, 2, R...><<<grid, CT_ROW_NT, ct_row_smem(), stream_>>>(
            reinterpret_cast<const cx<float> *>(post_), plane, W_, H_, plane_stride,
            reinterpret_cast<const cx<float> *>(ct_tw_row_), map);
        UPDC_CUDA(cudaGetLastError());
    }
    // S^T of the active exposures gathered straight into their scatter row
    // R2C (compile-time row transforms only): the scatter plane is not written.
    template <int... R> void launch_gather_row_r2c_ct(CtRadices<R...>) {
        dim3 grid((unsigned)ceil_div(H_, 2), (unsigned)act_n_);
        k_gather_row_r2c_ct<CT_ROW_NT, R...><<<grid, CT_ROW_NT, ct_row_smem(), stream_>>>(
            reinterpret_cast<const cx<float> *>(post_), reinterpret_cast<const ExpDesc<float> *>(d_exps_ + act_k0_),
            reinterpret_cast<const float *>(wr_ + (size_t)act_k0_ * nin_), nin_, W_, H_,
            reinterpret_cast<const cx<float> *>(ct_tw_row_), map_rs_);
        UPDC_CUDA(cudaGetLastError());
    }
    bool fused_gather() const { return ct_rows(); }
    void launch_gather_scatter_rows() {
        if constexpr (sizeof(T) == 4) ct_row_catalog(ct_row_rad_, [&](auto L) { launch_gather_row_r2c_ct(L); });
    }
    template <int... R> void launch_row_c2r_ct(CtRadices<R...>, int batch, float *out, const CUtensorMap &map) {
        dim3 grid((unsigned)ceil_div(H_, 2), (unsigned)batch);
        k_row_c2r_ct<CT_ROW_NT, 2, R...><<<grid, CT_ROW_NT, ct_row_smem(), stream_>>>(
            reinterpret_cast<const cx<float> *>(post_), map, H_, W_, (float)scale_factor(), out, nout_,
            reinterpret_cast<const cx<float> *>(ct_tw_row_), d_err_);
        UPDC_CUDA(cudaGetLastError());
    }
    template <class Acc> void configure_adjoint() {
        if constexpr (sizeof(typename Acc::S) > 0) {
            if constexpr (std::is_same<Acc, AccPlain<T>>::value || sizeof(T) == 4) {
                const size_t s = adj_smem<Acc>();
                by_pad(plan_h_.pad_shift, [&](auto P) {
                    constexpr int PS = decltype(P)::value;
                    set_smem(k_col_adjoint<T, Acc, ColNt<T>::value, Caps<T>::COL_S, ColAux<T>, PS>, s);
                    set_smem(k_col_adjoint<T, Acc, ColNt<T>::value, Caps<T>::COL_L, ColAux<T>, PS>, s);
                });
            }
        }
    }

    // ------------------------------------------------------------------ launches
    // planes [batch][H][W] -> u-major spectra [batch][M+1][ldh], one launch
    void launch_row_r2c_plane(const T *plane, cx<T> *out, int batch, size_t plane_stride, const CUtensorMap &map) {
        if (long_rows_) {
            long_r2c<T>(lrp_, PlaneLoader<T>{plane, W_, plane_stride}, W_, H_, batch, post_,
                        SpecRef{out, ldh_, (size_t)(M_ + 1) * ldh_}, long_scratch_);
            return;
        }
        if constexpr (sizeof(T) == 4) {
            if (ct_rows()) {
                ct_row_catalog(ct_row_rad_, [&](auto L) { launch_row_r2c_ct(L, plane, batch, plane_stride, map); });
                return;
            }
        }
        const int B = row_batch();
        dim3 grid((unsigned)ceil_div(H_, B), (unsigned)batch);
        const PlaneLoader<T> ld{plane, W_, plane_stride};
        const SpecRef ref{out, ldh_, (size_t)(M_ + 1) * ldh_};
        if constexpr (sizeof(T) == 4) {
            if (wide_rows_) {
                by_pad(plan_m_.pad_shift, [&](auto P) {
                    constexpr int PS = decltype(P)::value;
                    k_row_r2c<T, WIDE_NT, WIDE_CAP, PlaneLoader<T>, true, PS, 2><<<grid, WIDE_NT, row_smem(), stream_>>>(
                        plan_m_, post_, ld, W_, H_, 2, FastDiv(2u), ref, map);
                });
                UPDC_CUDA(cudaGetLastError());
                return;
            }
        }
        by_pad(plan_m_.pad_shift, [&](auto P) {
            by_rows(B, [&](auto Q) {
                constexpr int PS = decltype(P)::value, BR = decltype(Q)::value;
                if (use_tma_)
                    k_row_r2c<T, RowNt<T>::value, Caps<T>::ROW, PlaneLoader<T>, true, PS, BR><<<grid, RowNt<T>::value, row_smem(), stream_>>>(
                        plan_m_, post_, ld, W_, H_, B, FastDiv((uint32_t)B), ref, map);
                else
                    k_row_r2c<T, RowNt<T>::value, Caps<T>::ROW, PlaneLoader<T>, false, PS, BR><<<grid, RowNt<T>::value, row_smem(), stream_>>>(
                        plan_m_, post_, ld, W_, H_, B, FastDiv((uint32_t)B), ref, no_map_);
            });
        });
        UPDC_CUDA(cudaGetLastError());
    }
    void launch_col_forward() {
        if (long_cols_) return long_col_forward();
        const size_t nu = (size_t)M_ + 1;
        const size_t ks = nu * FH_, ys = nu * ldh_;
        if constexpr (sizeof(T) == 4) {
            if (ct_cols()) {
                ct_col_catalog(ct_col_rad_, [&](auto L) { launch_col_forward_ct(L); });
                return;
            }
        }
        by_pad(plan_h_.pad_shift, [&](auto P) {
            constexpr int PS = decltype(P)::value;
            if (FH_ <= Caps<T>::COL_S)
                k_col_forward<T, ColNt<T>::value, Caps<T>::COL_S, ColAux<T>, PS><<<(unsigned)nu, ColNt<T>::value, fwd_smem(), stream_>>>(plan_h_, rx_, ldh_, H_, khat_ + act_k0_ * ks, ks, act_n_, act_y(), ldh_, ys, H_, (int)nu, aux_fwd_);
            else
                k_col_forward<T, ColNt<T>::value, Caps<T>::COL_L, ColAux<T>, PS><<<(unsigned)nu, ColNt<T>::value, fwd_smem(), stream_>>>(plan_h_, rx_, ldh_, H_, khat_ + act_k0_ * ks, ks, act_n_, act_y(), ldh_, ys, H_, (int)nu, aux_fwd_);
        });
        UPDC_CUDA(cudaGetLastError());
    }
    template <int... R> void launch_col_forward_ct(CtRadices<R...>) {
        const size_t nu = (size_t)M_ + 1;
        const size_t ks = nu * FH_, ys = nu * ldh_;
        k_col_forward_ct<CT_COL_NT, R...><<<(unsigned)nu, CT_COL_NT, (size_t)FH_ * sizeof(cx<float>), stream_>>>(
            reinterpret_cast<const cx<float> *>(rx_), ldh_, H_,
            reinterpret_cast<const cx<float> *>(khat_ + act_k0_ * ks), ks, act_n_,
            reinterpret_cast<cx<float> *>(act_y()), ldh_, ys, H_, reinterpret_cast<cx<float> *>(aux_fwd_),
            reinterpret_cast<const cx<float> *>(ct_tw_col_));
        UPDC_CUDA(cudaGetLastError());
    }
    template <class Acc, int... R> void launch_col_adjoint_ct(CtRadices<R...>, const cx<T> *khat, typename Acc::S *aux) {
        const size_t nu = (size_t)M_ + 1;
        k_col_adjoint_ct<Acc, CT_COL_NT, R...><<<(unsigned)nu, CT_COL_NT, (size_t)FH_ * sizeof(cx<float>), stream_>>>(
            reinterpret_cast<const cx<float> *>(act_rs()), ldh_, nu * ldh_, H_,
            reinterpret_cast<const cx<float> *>(khat + act_k0_ * nu * FH_), nu * FH_, act_n_,
            reinterpret_cast<cx<float> *>(cr_), ldh_, H_, aux, reinterpret_cast<const cx<float> *>(ct_tw_col_));
        UPDC_CUDA(cudaGetLastError());
    }
    template <class Acc> void ensure_adj_aux() {
        if (adj_aux<Acc>() && !aux_adj_) aux_adj_ = alloc<typename Acc::S>(((size_t)M_ + 1) * FH_);
    }
    template <class Acc> void launch_col_adjoint_t(const cx<T> *khat) {
        const size_t nu = (size_t)M_ + 1;
        typename Acc::S *aux = nullptr;
        if (adj_aux<Acc>()) {
            if (!aux_adj_) aux_adj_ = alloc<typename Acc::S>(nu * FH_);
            aux = (typename Acc::S *)aux_adj_;
        }
        if constexpr (sizeof(T) == 4) {
            if (ct_cols() && aux) {
                ct_col_catalog(ct_col_rad_, [&](auto L) { launch_col_adjoint_ct<Acc>(L, khat, aux); });
                return;
            }
        }
        const size_t s = adj_smem<Acc>();
        by_pad(plan_h_.pad_shift, [&](auto P) {
            constexpr int PS = decltype(P)::value;
            if (FH_ <= Caps<T>::COL_S)
                k_col_adjoint<T, Acc, ColNt<T>::value, Caps<T>::COL_S, ColAux<T>, PS><<<(unsigned)nu, ColNt<T>::value, s, stream_>>>(plan_h_, act_rs(), ldh_, nu * ldh_, H_, khat + act_k0_ * nu * FH_, nu * FH_, act_n_, cr_, ldh_, H_, aux);
            else
                k_col_adjoint<T, Acc, ColNt<T>::value, Caps<T>::COL_L, ColAux<T>, PS><<<(unsigned)nu, ColNt<T>::value, s, stream_>>>(plan_h_, act_rs(), ldh_, nu * ldh_, H_, khat + act_k0_ * nu * FH_, nu * FH_, act_n_, cr_, ldh_, H_, aux);
        });
        UPDC_CUDA(cudaGetLastError());
    }
    void launch_col_adjoint() {
        if (long_cols_) {
            if constexpr (sizeof(T) == 4) {
                if (opt_.form == FORM_FP32) return long_col_adjoint<AccF64>(khat_);
                if (opt_.form == FORM_FP32_KAHAN) return long_col_adjoint<AccKahan>(khat_);
            }
            return long_col_adjoint<AccPlain<T>>(khat_);
        }
        if constexpr (sizeof(T) == 4) {
            if (opt_.form == FORM_FP32) return launch_col_adjoint_t<AccF64>(khat_);
            if (opt_.form == FORM_FP32_KAHAN) return launch_col_adjoint_t<AccKahan>(khat_);
        }
        launch_col_adjoint_t<AccPlain<T>>(khat_);
    }
    void launch_row_c2r_batched(const cx<T> *in, int batch, T *out, const CUtensorMap &map) {
        if (long_rows_) {
            long_c2r<T>(lrp_, post_, SpecRef{const_cast<cx<T> *>(in), ldh_, (size_t)(M_ + 1) * ldh_}, H_, batch, W_,
                        scale_factor(), PlaneStore<T>{out, W_, nout_}, long_scratch_);
            return;
        }
        if constexpr (sizeof(T) == 4) {
            if (ct_rows()) {
                ct_row_catalog(ct_row_rad_, [&](auto L) { launch_row_c2r_ct(L, batch, out, map); });
                return;
            }
        }
        const int B = row_batch();
        dim3 grid((unsigned)ceil_div(H_, B), (unsigned)batch);
        const T scale = scale_factor();
        const SpecRef ref{const_cast<cx<T> *>(in), ldh_, (size_t)(M_ + 1) * ldh_};
        if constexpr (sizeof(T) == 4) {
            if (wide_rows_) {
                by_pad(plan_m_.pad_shift, [&](auto P) {
                    constexpr int PS = decltype(P)::value;
                    k_row_c2r<T, WIDE_NT, WIDE_CAP, PlaneStore<T>, true, PS, 2><<<grid, WIDE_NT, row_smem(), stream_>>>(
                        plan_m_, post_, ref, map, H_, W_, 2, FastDiv(2u), scale, PlaneStore<T>{out, W_, nout_}, d_err_);
                });
                UPDC_CUDA(cudaGetLastError());
                return;
            }
        }
        by_pad(plan_m_.pad_shift, [&](auto P) {
            by_rows(B, [&](auto Q) {
                constexpr int PS = decltype(P)::value, BR = decltype(Q)::value;
                if (use_tma_)
                    k_row_c2r<T, RowNt<T>::value, Caps<T>::ROW, PlaneStore<T>, true, PS, BR><<<grid, RowNt<T>::value, row_smem(), stream_>>>(
                        plan_m_, post_, ref, map, H_, W_, B, FastDiv((uint32_t)B), scale, PlaneStore<T>{out, W_, nout_}, d_err_);
                else
                    k_row_c2r<T, RowNt<T>::value, Caps<T>::ROW, PlaneStore<T>, false, PS, BR><<<grid, RowNt<T>::value, row_smem(), stream_>>>(
                        plan_m_, post_, ref, no_map_, H_, W_, B, FastDiv((uint32_t)B), scale, PlaneStore<T>{out, W_, nout_}, d_err_);
            });
        });
        UPDC_CUDA(cudaGetLastError());
    }
    T scale_factor() const {
        // updc_core.c:741 scale = 1.0f/(float)nf
        if (sizeof(T) == 4) return (T)(1.0f / (float)((size_t)FW_ * FH_));
        return (T)(1.0 / (double)((size_t)FW_ * FH_));
    }
    void launch_detector() {
        dim3 grid((unsigned)std::min<size_t>(ceil_div(nin_, 256), 148 * 8), (unsigned)act_n_);
        const size_t k0 = act_k0_;
        if (comp_mu_)
            k_detector<T, true><<<grid, 256, sizeof(DetShared), stream_>>>(d_exps_ + k0, nin_, nout_, blur_ + k0 * nout_, wr_ + k0 * nin_,
                                                            d_stats_ + k0, d_err_);
        else
            k_detector<T, false><<<grid, 256, sizeof(DetShared), stream_>>>(d_exps_ + k0, nin_, nout_, blur_ + k0 * nout_, wr_ + k0 * nin_,
                                                             d_stats_ + k0, d_err_);
        UPDC_CUDA(cudaGetLastError());
    }
    void launch_scatter(const T *vals, T *out) {
        dim3 grid((unsigned)std::min<size_t>(ceil_div(nout_, 256), 148 * 8), (unsigned)act_n_);
        const size_t k0 = act_k0_;
        k_scatter_t<T, T, T><<<grid, 256, 0, stream_>>>(d_exps_ + k0, nin_, nout_, vals + k0 * nin_, 0, out + k0 * nout_);
        UPDC_CUDA(cudaGetLastError());
    }
    void launch_update() {
        k_update_vec<T><<<upd_grid_, 256, 0, stream_>>>(nout_, correction_, den_, estimate_, max_sens_, d_err_, d_part_sum_,
                                                        d_part_neg_, d_upd_done_, d_red_sum_, d_red_neg_);
        UPDC_CUDA(cudaGetLastError());
    }
    // The per-iteration counters' initial values (nnew = ntotal = 0, min =
    // ~0), kept on the device so that an iteration enqueues only copies
    // (nothing allocates or waits inside a stream capture).
    void init_stats_template() {
        static_assert(sizeof(ExpStats) == 32, "ExpStats layout");
        std::vector<ExpStats> init(nexp_);
        for (auto &s : init) { s.nnew = 0; s.ntotal = 0; s.min_ordered = ~0ull; s.pad = 0; }
        stats_init_ = alloc<ExpStats>(nexp_);
        UPDC_CUDA(cudaMemcpy(stats_init_, init.data(), nexp_ * sizeof(ExpStats), cudaMemcpyHostToDevice));
    }
    void reset_iteration_state() {
        UPDC_CUDA(cudaMemcpyAsync(d_stats_, stats_init_, nexp_ * sizeof(ExpStats), cudaMemcpyDeviceToDevice, stream_));
        UPDC_CUDA(cudaMemsetAsync(d_err_, 0xFF, 8, stream_));
    }
    ExpStats *stats_init_ = nullptr;

    // The launches of one iteration; mark(i) is called at the stage
    // boundaries (events of the stage timing), the update only with `update`.
    template <class Mark> void enqueue_stages(const Mark &mark, bool update) {
        mark(0);
        reset_iteration_state();
        launch_row_r2c_plane(estimate_, rx_, 1, 0, map_rx_);                      // estimate R2C, x pass
        mark(1);
        launch_col_forward();                                               // y pass + OTF + inverse y pass
        mark(2);
        launch_row_c2r_batched(act_y(), act_n_, blur_ + (size_t)act_k0_ * nout_, map_y_);  // inverse x pass + crop
        mark(3);
        launch_detector();                                                  // gather / FreezeMu / ratio
        mark(4);
        if (fused_gather()) {
            // S^T gathered inside the scatter R2C's x pass (timed as that pass)
            mark(5);
            launch_gather_scatter_rows();
        } else {
            launch_scatter(wr_, scatter_);                                  // S^T (transposed gather)
            mark(5);
            launch_row_r2c_plane(scatter_ + (size_t)act_k0_ * nout_, act_rs(), act_n_, nout_, map_rs_);  // scatter R2C, x pass
        }
        mark(6);
        launch_col_adjoint();                                               // y pass, conj-OTF sum, inverse y
        launch_row_c2r_batched(cr_, 1, correction_, map_cr_);                        // inverse x pass + crop
        mark(7);
        if (update) launch_update();
        mark(8);
    }
    void enqueue_iteration(bool timed) {
        if (!timed) return enqueue_stages([](int) {}, true);
        cudaEvent_t ev[9];
        for (auto &e : ev) UPDC_CUDA(cudaEventCreate(&e));
        enqueue_stages([&](int i) { UPDC_CUDA(cudaEventRecord(ev[i], stream_)); }, true);
        UPDC_CUDA(cudaEventSynchronize(ev[8]));
        for (int s = 0; s < 8; ++s) UPDC_CUDA(cudaEventElapsedTime(&stage_ms_[s], ev[s], ev[s + 1]));
        for (auto &e : ev) cudaEventDestroy(e);
    }

    // One iteration with its events and the copies of its record into
    // pinned slot i (stats, error key, signed sum, negative count).  Inside a
    // capture the events become external event-record nodes, so they keep
    // their timestamps when the graph runs.
    void enqueue_recorded(int i, bool graph, bool capturing = false) {
        const size_t rec_bytes = rec_stride();
        const unsigned flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
        UPDC_CUDA(cudaEventRecordWithFlags(events_[2 * i], stream_, flags));
        if (graph) UPDC_CUDA(cudaGraphLaunch(graph_exec_, stream_));
        else enqueue_iteration(opt_.stage_timing != 0);
        UPDC_CUDA(cudaEventRecordWithFlags(events_[2 * i + 1], stream_, flags));
        char *dst = (char *)pinned_ + (size_t)i * rec_bytes;
        UPDC_CUDA(cudaMemcpyAsync(dst, d_stats_, nexp_ * sizeof(ExpStats), cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaMemcpyAsync(dst + nexp_ * sizeof(ExpStats), d_err_, 8, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaMemcpyAsync(dst + nexp_ * sizeof(ExpStats) + 8, d_red_sum_, 8, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaMemcpyAsync(dst + nexp_ * sizeof(ExpStats) + 16, d_red_neg_, 8, cudaMemcpyDeviceToHost, stream_));
    }

    // Graph of n whole iterations (cached per n; rebuilt if the pinned
    // record buffer moves).
    static constexpr int LOOP_GRAPH_MAX = 256;
    std::map<int, cudaGraphExec_t> loop_graphs_;
    void drop_loop_graphs() {
        for (auto &g : loop_graphs_) cudaGraphExecDestroy(g.second);
        loop_graphs_.clear();
    }
    cudaGraphExec_t loop_graph(int n) {
        auto it = loop_graphs_.find(n);
        if (it != loop_graphs_.end()) return it->second;
        if (loop_graphs_.size() >= 8) drop_loop_graphs();
        reset_iteration_state();
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        cudaGraph_t g = nullptr;
        UPDC_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            for (int i = 0; i < n; ++i) enqueue_recorded(i, false, true);
        } catch (...) {
            cudaStreamEndCapture(stream_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        UPDC_CUDA(cudaStreamEndCapture(stream_, &g));
        cudaGraphExec_t ex = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        UPDC_CUDA(e);
        loop_graphs_[n] = ex;
        return ex;
    }

    void build_graph() {
        // the stats-initialiser buffer must exist before capture
        reset_iteration_state();
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        UPDC_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_iteration(false);
        } catch (...) {
            // end the capture, or every later call of this thread fails
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        UPDC_CUDA(cudaStreamEndCapture(stream_, &graph_));
        UPDC_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0));
    }

    [[noreturn]] void raise_device_error(unsigned long long key) {
        const uint32_t code = (uint32_t)(key & 0xFF);
        const uint64_t index = (key >> 8) & 0xFFFFFFFFFFull;
        std::string detail;
        if (code == ERR_NEGATIVE_CORRECTION && index < nout_) {
            T c = 0, d = 0;
            UPDC_CUDA(cudaMemcpy(&c, correction_ + index, sizeof(T), cudaMemcpyDeviceToHost));
            UPDC_CUDA(cudaMemcpy(&d, den_ + index, sizeof(T), cudaMemcpyDeviceToHost));
            char buf[256];
            snprintf(buf, sizeof(buf), "negative correction at target %llu: C=%.9g numerator=%.9g denominator=%.9g\n",
                     (unsigned long long)index, (double)(c / d), (double)c, (double)d);
            fputs(buf, stderr);
        }
        throw Error(1, error_message(code));
    }
    void check_error() {
        unsigned long long key;
        UPDC_CUDA(cudaMemcpy(&key, d_err_, 8, cudaMemcpyDeviceToHost));
        if (key != ~0ull) raise_device_error(key);
    }

    const void *plane_ptr(int which, int k, size_t *n) {
        *n = nout_;
        switch (which) {
            case PLANE_ESTIMATE: return estimate_;
            case PLANE_COVERAGE: return coverage_;
            case PLANE_DENOMINATOR: return den_;
            case PLANE_CORRECTION: return correction_;
            case PLANE_BLUR: return blur_ + (size_t)k * nout_;
            case PLANE_SCATTER: return scatter_ + (size_t)k * nout_;
            case PLANE_SCIENCE: *n = nin_; return sci_ + (size_t)k * nin_;
            case PLANE_WEIGHT: *n = nin_; return wht_ + (size_t)k * nin_;
            case PLANE_WR: *n = nin_; return wr_ + (size_t)k * nin_;
            case PLANE_FROZEN: *n = nin_; return frozen_ + (size_t)k * nin_;
            default: throw Error(1, "unknown plane");
        }
    }

    // ------------------------------------------------------------------ setup stages
    void prepare_links(int k) {
        ExposureInput &e = exps_[k];
        DevLinkMap &m = links_[k];
        bool ok = opt_.reuse_links && linkmap_load(e.links, nin_, W_, H_, m, stream_);
        if (!ok) {
            LinkBuildStats st;
            linkmap_build(e.vertices, e.links, iw_, ih_, W_, H_, stream_, &st);
            if (opt_.verbose)
                printf("AreaLink exposure %d: %llu overlaps; encoding=%s; active=%llu, max-links=%u (GPU)\n", k + 1,
                       (unsigned long long)st.nlinks, st.encoding == LINKMAP_DELTA16 ? "DELTA16" : "ABS32",
                       (unsigned long long)st.active, st.max_links);
            if (!linkmap_load(e.links, nin_, W_, H_, m, stream_)) throw Error(1, "invalid or obsolete LinkMap cache");
        } else if (opt_.verbose) {
            printf("AreaLink exposure %d: persistent cache hit (%s)\n", k + 1,
                   m.encoding == LINKMAP_DELTA16 ? "DELTA16" : "ABS32");
        }
        linkmap_transpose(m, nout_, stream_);
        bytes_ += m.file_bytes - 64 + (nout_ + 1) * 4 + m.nlinks * 8;
    }

    void upload_descs() {
        std::vector<ExpDesc<T>> h(nexp_);
        for (int k = 0; k < nexp_; ++k) {
            const DevLinkMap &m = links_[k];
            ExpDesc<T> &d = h[k];
            d.off = m.off; d.base = m.base; d.tgt = m.tgt; d.delta = m.delta; d.frac = m.frac;
            d.toff = m.toff; d.tent = m.tent;
            d.sci = sci_ + (size_t)k * nin_;
            d.wht = wht_ + (size_t)k * nin_;
            d.frozen = frozen_ + (size_t)k * nin_;
            const ExposureInput &e = exps_[k];
            if (sizeof(T) == 4) {
                d.background = (T)e.backgroundf;
                d.pedestal = (T)e.pedestalf;
                d.mean_offset = (T)(e.backgroundf + e.pedestalf);
            } else {
                d.background = (T)e.background;
                d.pedestal = (T)e.pedestal;
                d.mean_offset = (T)(e.background + e.pedestal);
            }
            d.delta16 = m.encoding == LINKMAP_DELTA16;
        }
        UPDC_CUDA(cudaMemcpy(d_exps_, h.data(), nexp_ * sizeof(ExpDesc<T>), cudaMemcpyHostToDevice));
    }

    void load_planes() {
        float *h = nullptr;
        UPDC_CUDA(cudaMallocHost(&h, 2 * nin_ * sizeof(float)));
        float *d_raw = dalloc<float>(2 * nin_ * nexp_, nullptr);
        // every 64th weight of every exposure, finite and > 0 (updc_core.c:379-386)
        float *d_sample = dalloc<float>(nexp_ * (nin_ / 64 + 1) + 1, nullptr);
        unsigned int *d_count = dalloc<unsigned int>(1, nullptr);
        UPDC_CUDA(cudaMemset(d_count, 0, 4));
        for (int k = 0; k < nexp_; ++k) {
            if (!read_f32_exact(exps_[k].science, h, nin_)) { cudaFreeHost(h); throw Error(1, "cannot read SCI raw: " + exps_[k].science); }
            if (!read_f32_exact(exps_[k].weight, h + nin_, nin_)) { cudaFreeHost(h); throw Error(1, "cannot read WHT raw: " + exps_[k].weight); }
            UPDC_CUDA(cudaMemcpy(d_raw + 2 * nin_ * k, h, 2 * nin_ * sizeof(float), cudaMemcpyHostToDevice));
            k_weight_sample<<<grid1d(nin_ / 64 + 1), 256, 0, stream_>>>(nin_, d_raw + 2 * nin_ * k + nin_, d_sample, d_count);
        }
        unsigned int n = 0;
        UPDC_CUDA(cudaMemcpyAsync(&n, d_count, 4, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        cudaFreeHost(h);
        if (!n) throw Error(1, "all input WHT pixels are zero");
        // median sample[n/2] of the sorted samples (positive floats sort as their bits)
        float *d_sorted = dalloc<float>(n, nullptr);
        size_t tmp_bytes = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, (const uint32_t *)d_sample, (uint32_t *)d_sorted, (int)n, 0, 32, stream_);
        void *tmp = dalloc<char>(tmp_bytes, nullptr);
        cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, (const uint32_t *)d_sample, (uint32_t *)d_sorted, (int)n, 0, 32, stream_);
        float scale = 0;
        UPDC_CUDA(cudaMemcpyAsync(&scale, d_sorted + n / 2, 4, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(tmp);
        cudaFree(d_sorted);
        cudaFree(d_sample);
        if (!(scale > 0) || !std::isfinite(scale)) { cudaFree(d_raw); cudaFree(d_count); throw Error(1, "invalid WHT normalization"); }
        weight_scale_ = (T)scale;
        unsigned long long *d_masked = dalloc<unsigned long long>(1, nullptr);
        UPDC_CUDA(cudaMemset(d_masked, 0, 8));
        UPDC_CUDA(cudaMemset(d_err_, 0xFF, 8));
        for (int k = 0; k < nexp_; ++k) {
            const T ped = sizeof(T) == 4 ? (T)exps_[k].pedestalf : (T)exps_[k].pedestal;
            k_weight_norm<T><<<grid1d(nin_), 256, 0, stream_>>>(nin_, d_raw + 2 * nin_ * k, d_raw + 2 * nin_ * k + nin_,
                                                                 sci_ + (size_t)k * nin_, wht_ + (size_t)k * nin_,
                                                                 weight_scale_, ped, k, d_masked, d_err_);
        }
        UPDC_CUDA(cudaGetLastError());
        unsigned long long hm = 0;
        UPDC_CUDA(cudaMemcpyAsync(&hm, d_masked, 8, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        masked_ = hm;
        cudaFree(d_masked);
        cudaFree(d_raw);
        cudaFree(d_count);
        check_error();
        upload_descs();
    }

    // PSF spectra K_k (u-major, (M+1) x FH) of precision U into dst.
    template <typename U>
    void psf_spectra(cx<U> *dst, bool fp64_sum, const FftPlan &pm, const FftPlan &ph, const cx<U> *post) {
        const size_t nu = (size_t)M_ + 1;
        cx<U> *rp = dalloc<cx<U>>(nu * FH_, nullptr);
        try {
            for (int k = 0; k < nexp_; ++k) {
                if (!active(k)) continue;
                const ExposureInput &e = exps_[k];
                const size_t count = (size_t)e.psf_width * e.psf_height;
                std::vector<float> hp(count);
                if (!read_f32_exact(e.psf, hp.data(), count)) throw Error(1, "cannot read PSF raw: " + e.psf);
                psf_spectrum_one<U, float>(hp.data(), e.psf_width, e.psf_height, dst + (size_t)k * nu * FH_, rp,
                                           fp64_sum, pm, ph, post);
            }
        } catch (...) {
            cudaFree(rp);
            throw;
        }
        cudaFree(rp);
    }

    // One PSF (host array, manifest layout) to its spectrum `out`: sum (FP64,
    // or the reference's Neumaier FP32), 1/sum, centre wrap, R2C
    // (prepare_psf_with_buffers, updc_core.c:777-843).  `rp` is an
    // (M+1) x FH scratch.  An FP64 PSF (differentiable model) is summed in FP64.
    template <typename U, typename P>
    void psf_spectrum_one(const P *hp, int pw, int phh, cx<U> *out, cx<U> *rp, bool fp64_sum, const FftPlan &pm,
                          const FftPlan &ph, const cx<U> *post) {
        const size_t nu = (size_t)M_ + 1;
        const size_t count = (size_t)pw * phh;
        if (sizeof(P) == 8) fp64_sum = true;
        P *dp = dalloc<P>(count, nullptr);
        try {
            UPDC_CUDA(cudaMemcpy(dp, hp, count * sizeof(P), cudaMemcpyHostToDevice));
            UPDC_CUDA(cudaMemset(d_err_, 0xFF, 8));
            double sum = 0;
            if (fp64_sum) {
                const int g = 148;
                double *part = dalloc<double>(g, nullptr);
                k_psf_sum_f64<P><<<g, 256, 0, stream_>>>(dp, count, part, d_err_);
                std::vector<double> hpart(g);
                UPDC_CUDA(cudaMemcpyAsync(hpart.data(), part, g * 8, cudaMemcpyDeviceToHost, stream_));
                UPDC_CUDA(cudaStreamSynchronize(stream_));
                for (double v : hpart) sum += v;
                cudaFree(part);
            } else {
                float *ds = dalloc<float>(1, nullptr);
                k_psf_sum_neumaier<<<1, 1, 0, stream_>>>((const float *)dp, count, ds, d_err_);
                float hs = 0;
                UPDC_CUDA(cudaMemcpyAsync(&hs, ds, 4, cudaMemcpyDeviceToHost, stream_));
                UPDC_CUDA(cudaStreamSynchronize(stream_));
                sum = hs;
                cudaFree(ds);
            }
            check_error();
            if (!(sum > 0) || !std::isfinite(sum)) throw Error(1, "PSF sum is zero/non-finite");
            U inv;
            if (fp64_sum) inv = (U)(1.0 / sum);
            else inv = (U)(1.0f / (float)sum);
            PsfLoader<U, P> ld{dp, pw, transposed_ ? phh : pw, transposed_ ? pw : phh, FW_, FH_, transposed_, inv};
            if (long_rows_) {
                // four-step rows; a temporary plan and scratch of precision U
                std::vector<void *> owned;
                auto get = [&](size_t n) {
                    owned.push_back(dalloc<cx<U>>(n, nullptr));
                    return owned.back();
                };
                try {
                    const LongRowPlan lp = make_long_plan<U>(lrp_.M1, lrp_.M2, get);
                    cx<U> *scr = (cx<U> *)get((size_t)FH_ * M_);
                    long_r2c<U>(lp, ld, FW_, FH_, 1, post, SpecRef{rp, FH_, 0}, scr);
                    col_fft_psf<U>(ph, rp, out);
                    UPDC_CUDA(cudaStreamSynchronize(stream_));
                } catch (...) {
                    for (void *q : owned) cudaFree(q);
                    throw;
                }
                for (void *q : owned) cudaFree(q);
                cudaFree(dp);
                return;
            }
            const int B = Caps<U>::ROW / M_;
            const size_t rsm = row_buf_bytes(B, M_, sizeof(cx<U>), pm.pad_shift);
            set_smem(k_row_r2c<U, RowNt<U>::value, Caps<U>::ROW, PsfLoader<U, P>, false>, rsm);
            dim3 grid((unsigned)ceil_div(FH_, B), 1);
            k_row_r2c<U, RowNt<U>::value, Caps<U>::ROW, PsfLoader<U, P>, false><<<grid, RowNt<U>::value, rsm, stream_>>>(
                pm, post, ld, FW_, FH_, B, FastDiv((uint32_t)B), SpecRef{rp, FH_, 0}, no_map_);
            col_fft_psf<U>(ph, rp, out);
            UPDC_CUDA(cudaStreamSynchronize(stream_));
        } catch (...) {
            cudaFree(dp);
            throw;
        }
        cudaFree(dp);
    }

    void prepare_psf_spectra() {
        const bool fp64_sum = opt_.form == FORM_FP32 || opt_.form == FORM_FP64;
        psf_spectra<T>(khat_, fp64_sum, plan_m_, plan_h_, post_);
    }

    void drizzle() {
        if (shard_setup_) {
            k_drizzle_partial<T><<<grid1d(nout_), 256, 0, stream_>>>(d_exps_ + act_k0_, act_n_, nout_, coverage_, estimate_,
                                                                    correction_);
            UPDC_CUDA(cudaGetLastError());
            UPDC_CUDA(cudaStreamSynchronize(stream_));
            return;
        }
        UPDC_CUDA(cudaMemset(d_err_, 0xFF, 8));
        k_drizzle<T><<<grid1d(nout_), 256, 0, stream_>>>(d_exps_, nexp_, nout_, estimate_, coverage_, d_err_);
        UPDC_CUDA(cudaGetLastError());
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        check_error();
    }

    // D = crop(C2R(sum_k conj(K_k) R2C(pad(S_k^T W_k)))) / nf   (updc_core.c:1026-1086)
    void denominator() {
        // the active exposures' terms (all of them unless this is a shard set up alone)
        if (sizeof(T) == 4 && opt_.form == FORM_FP32) denominator_fp64();
        else {
            dim3 grid((unsigned)std::min<size_t>(ceil_div(nout_, 256), 148 * 8), (unsigned)act_n_);
            k_scatter_t<T, T, T><<<grid, 256, 0, stream_>>>(d_exps_ + act_k0_, nin_, nout_, (const T *)nullptr, 1,
                                                            scatter_ + (size_t)act_k0_ * nout_);
            launch_row_r2c_plane(scatter_ + (size_t)act_k0_ * nout_, act_rs(), act_n_, nout_, map_rs_);
            launch_col_adjoint();
            launch_row_c2r_batched(cr_, 1, den_, map_cr_);
        }
        if (shard_setup_) UPDC_CUDA(cudaStreamSynchronize(stream_));
        else finish_denominator();
    }

    // Column FFTs of the PSF's row-pass output rp ((M+1) x FH) into out.
    template <typename U> void col_fft_psf(const FftPlan &ph, const cx<U> *rp, cx<U> *out) {
        const size_t nu = (size_t)M_ + 1;
        if (long_cols_) {
            // four-step columns: a temporary plan and scratch of precision U
            std::vector<void *> owned;
            auto get = [&](size_t n) {
                owned.push_back(dalloc<cx<U>>(n, nullptr));
                return owned.back();
            };
            try {
                const LongColPlan lp = col_plan(make_long_plan<U>(lcp_.N1, lcp_.N2, get));
                cx<U> *scr = (cx<U> *)get(nu * FH_);
                long_col_fft<U, false>(lp, rp, FH_, FH_, out, FH_, FH_, (int)nu, scr);
                UPDC_CUDA(cudaStreamSynchronize(stream_));
            } catch (...) {
                for (void *q : owned) cudaFree(q);
                throw;
            }
            for (void *q : owned) cudaFree(q);
            return;
        }
        const size_t cs = fft_buf_bytes(FH_, sizeof(cx<U>), ph.pad_shift);
        if (FH_ <= Caps<U>::COL_S) {
            set_smem(k_col_fft<U, NT, Caps<U>::COL_S, false>, cs);
            k_col_fft<U, NT, Caps<U>::COL_S, false><<<(unsigned)nu, NT, cs, stream_>>>(ph, rp, FH_, FH_, out, FH_, FH_);
        } else {
            set_smem(k_col_fft<U, NT, Caps<U>::COL_L, false>, cs);
            k_col_fft<U, NT, Caps<U>::COL_L, false><<<(unsigned)nu, NT, cs, stream_>>>(ph, rp, FH_, FH_, out, FH_, FH_);
        }
        UPDC_CUDA(cudaGetLastError());
    }

    // FP32 form: the one-time denominator is computed entirely in FP64.
    void denominator_fp64() {
        using D = double;
        const size_t nu = (size_t)M_ + 1;
        FftPlan pm, ph;
        auto tm = fft_make_table<D>(M_, FFT_RMAX, pm);
        auto th = fft_make_table<D>(FH_, FFT_RMAX, ph);
        pm.pad_shift = fft_choose_padding(pm, NT, Caps<D>::ROW, std::max(1, std::min(2, Caps<D>::ROW / M_)));
        ph.pad_shift = fft_choose_padding(ph, NtAdj<D>::value, Caps<D>::COL_S, 1);
        cx<D> *dm = dalloc<cx<D>>(tm.size(), nullptr), *dh = dalloc<cx<D>>(th.size(), nullptr);
        UPDC_CUDA(cudaMemcpy(dm, tm.data(), tm.size() * sizeof(cx<D>), cudaMemcpyHostToDevice));
        UPDC_CUDA(cudaMemcpy(dh, th.data(), th.size() * sizeof(cx<D>), cudaMemcpyHostToDevice));
        pm.tw = dm;
        ph.tw = dh;
        std::vector<cx<D>> post(M_ + 1);
        const double two_pi = 6.283185307179586476925286766559;
        for (int u = 0; u <= M_; ++u) post[u] = cx<D>{std::cos(-two_pi * u / FW_), std::sin(-two_pi * u / FW_)};
        cx<D> *dpost = dalloc<cx<D>>(M_ + 1, nullptr);
        UPDC_CUDA(cudaMemcpy(dpost, post.data(), post.size() * sizeof(cx<D>), cudaMemcpyHostToDevice));
        cx<D> *kd = dalloc<cx<D>>(nexp_ * nu * FH_, nullptr);
        psf_spectra<D>(kd, true, pm, ph, dpost);
        D *sc = dalloc<D>(nexp_ * nout_, nullptr);
        // the active exposures' terms (all of them unless this is a shard set up alone)
        dim3 grid((unsigned)std::min<size_t>(ceil_div(nout_, 256), 148 * 8), (unsigned)act_n_);
        k_scatter_t<T, D, T><<<grid, 256, 0, stream_>>>(d_exps_ + act_k0_, nin_, nout_, (const T *)nullptr, 1, sc);
        cx<D> *rs = dalloc<cx<D>>(nexp_ * nu * H_, nullptr), *cr = dalloc<cx<D>>(nu * H_, nullptr);
        const int B = std::max(1, Caps<D>::ROW / M_);
        const size_t rsm = row_buf_bytes(B, M_, sizeof(cx<D>), pm.pad_shift);
        // long rows: an FP64 four-step plan and its scratch, freed below
        std::vector<void *> lowned;
        LongRowPlan lpd;
        cx<D> *lscr = nullptr;
        if (long_rows_) {
            auto get = [&](size_t n) {
                lowned.push_back(dalloc<cx<D>>(n, nullptr));
                return lowned.back();
            };
            lpd = make_long_plan<D>(lrp_.M1, lrp_.M2, get);
            lscr = (cx<D> *)get((size_t)nexp_ * H_ * M_);
            long_r2c<D>(lpd, PlaneLoader<D>{sc, W_, nout_}, W_, H_, act_n_, dpost, SpecRef{rs, H_, nu * H_}, lscr);
        } else {
            set_smem(k_row_r2c<D, RowNt<D>::value, Caps<D>::ROW, PlaneLoader<D>, false>, rsm);
            dim3 g((unsigned)ceil_div(H_, B), (unsigned)act_n_);
            k_row_r2c<D, RowNt<D>::value, Caps<D>::ROW, PlaneLoader<D>, false><<<g, RowNt<D>::value, rsm, stream_>>>(
                pm, dpost, PlaneLoader<D>{sc, W_, nout_}, W_, H_, B, FastDiv((uint32_t)B), SpecRef{rs, H_, nu * H_}, no_map_);
        }
        const size_t b = fft_buf_bytes(FH_, sizeof(cx<D>), ph.pad_shift);
        const bool aux_needed = b + align16(FH_ * sizeof(cx<D>)) > SMEM_LIMIT;
        cx<D> *aux = aux_needed ? dalloc<cx<D>>(nu * FH_, nullptr) : nullptr;
        const size_t s = aux_needed ? b : b + align16(FH_ * sizeof(cx<D>));
        if (long_cols_) {
            // four-step FP64 columns: temporary plan, scratch, product and sum planes
            auto get = [&](size_t n) {
                lowned.push_back(dalloc<cx<D>>(n, nullptr));
                return lowned.back();
            };
            const LongColPlan lc = col_plan(make_long_plan<D>(lcp_.N1, lcp_.N2, get));
            const size_t n = nu * FH_;
            cx<D> *cs = (cx<D> *)get(n), *tmp = (cx<D> *)get(n), *sum = (cx<D> *)get(n);
            for (int j = 0; j < act_n_; ++j) {
                long_col_fft<D, false>(lc, rs + (size_t)j * nu * H_, H_, H_, tmp, FH_, FH_, (int)nu, cs);
                k_long_acc<D, AccPlain<D>><<<grid1d(n), 256, 0, stream_>>>(tmp, kd + (size_t)(act_k0_ + j) * n, sum, n,
                                                                           j == 0);
            }
            long_col_fft<D, true>(lc, sum, FH_, FH_, cr, H_, H_, (int)nu, cs);
        } else if (FH_ <= Caps<D>::COL_S) {
            set_smem(k_col_adjoint<D, AccPlain<D>, NtAdj<D>::value,Caps<D>::COL_S>, s);
            k_col_adjoint<D, AccPlain<D>, NtAdj<D>::value,Caps<D>::COL_S><<<(unsigned)nu, NtAdj<D>::value, s, stream_>>>(ph, rs, H_, nu * H_, H_, kd + (size_t)act_k0_ * nu * FH_, nu * FH_, act_n_, cr, H_, H_, aux);
        } else {
            set_smem(k_col_adjoint<D, AccPlain<D>, NtAdj<D>::value,Caps<D>::COL_L>, s);
            k_col_adjoint<D, AccPlain<D>, NtAdj<D>::value,Caps<D>::COL_L><<<(unsigned)nu, NtAdj<D>::value, s, stream_>>>(ph, rs, H_, nu * H_, H_, kd + (size_t)act_k0_ * nu * FH_, nu * FH_, act_n_, cr, H_, H_, aux);
        }
        D *den = dalloc<D>(nout_, nullptr);
        if (long_rows_) {
            long_c2r<D>(lpd, dpost, SpecRef{cr, H_, 0}, H_, 1, W_, 1.0 / (double)((size_t)FW_ * FH_),
                        PlaneStore<D>{den, W_, 0}, lscr);
        } else {
            set_smem(k_row_c2r<D, RowNt<D>::value, Caps<D>::ROW, PlaneStore<D>, false>, rsm);
            dim3 g2((unsigned)ceil_div(H_, B), 1);
            k_row_c2r<D, RowNt<D>::value, Caps<D>::ROW, PlaneStore<D>, false><<<g2, RowNt<D>::value, rsm, stream_>>>(
                pm, dpost, SpecRef{cr, H_, 0}, no_map_, H_, W_, B, FastDiv((uint32_t)B), 1.0 / (double)((size_t)FW_ * FH_),
                PlaneStore<D>{den, W_, 0}, d_err_);
        }
        k_convert<D, T><<<grid1d(nout_), 256, 0, stream_>>>(den, den_, nout_);
        UPDC_CUDA(cudaGetLastError());
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        for (void *p : {(void *)dm, (void *)dh, (void *)dpost, (void *)kd, (void *)sc, (void *)rs, (void *)cr, (void *)aux, (void *)den})
            if (p) cudaFree(p);
        for (void *p : lowned) cudaFree(p);
    }

    void finish_denominator() {
        unsigned long long *d = dalloc<unsigned long long>(1, nullptr);
        UPDC_CUDA(cudaMemset(d, 0, 8));
        k_max_ordered<T><<<grid1d(nout_), 256, 0, stream_>>>(den_, nout_, d);
        unsigned long long h = 0;
        UPDC_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, stream_));
        UPDC_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(d);
        double m = h ? ordered_to_double(h) : 0.0;
        if (!(m > 0)) m = 0;  // the reference starts its maximum at 0
        max_sens_ = (T)m;
        if (!(max_sens_ > 0) || !std::isfinite((double)max_sens_)) throw Error(1, "invalid H^T W sensitivity");
    }
};

}  // namespace

// ---------------------------------------------------------------------------- wait-timeout check
// A bounded mbarrier wait that must run out: thread 0 arms the barrier with
// an expected transaction count that no copy will ever deliver (nothing is
// issued, so nothing is in flight), every thread polls it at most `polls`
// times, and the block decides together (as the row kernels do) to record
// ERR_DEVICE_TIMEOUT and return.  The same path a stuck TMA tile takes.
__global__ void k_wait_timeout_probe(uint32_t polls, unsigned long long *err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, 16);
    }
    __syncthreads();
    const bool arrived = mbar_wait_bounded(&bar, 0, polls);
    if (__syncthreads_or(!arrived)) {
        if (threadIdx.x == 0) atomicMin(err, (unsigned long long)make_error_key(STAGE_TRANSFORM, 0, ERR_DEVICE_TIMEOUT));
        return;
    }
}

void device_wait_check(uint32_t polls) {
    unsigned long long *err = nullptr;
    cudaStream_t s = nullptr;
    UPDC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    UPDC_CUDA(cudaMalloc(&err, 8));
    unsigned long long key = ~0ull;
    UPDC_CUDA(cudaMemsetAsync(err, 0xFF, 8, s));
    k_wait_timeout_probe<<<1, 32, 0, s>>>(polls, err);
    cudaError_t rc = cudaGetLastError();
    if (rc == cudaSuccess) rc = cudaMemcpyAsync(&key, err, 8, cudaMemcpyDeviceToHost, s);
    if (rc == cudaSuccess) rc = cudaStreamSynchronize(s);
    cudaFree(err);
    cudaStreamDestroy(s);
    UPDC_CUDA(rc);
    if (key != ~0ull) throw Error(1, error_message((uint32_t)(key & 0xFF)));
}

std::unique_ptr<Engine> make_engine(const EngineOptions &opt) {
    if (opt.form == FORM_FP64) return std::unique_ptr<Engine>(new EngineImpl<double>(opt));
    return std::unique_ptr<Engine>(new EngineImpl<float>(opt));
}

}  // namespace updc
