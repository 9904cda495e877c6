// Batched fields: many independent UPDC fields of uneven grid size and
// exposure count iterated together.  Each field is set up by its own engine
// (FFT shape and autotuned radix splits, LinkMaps, PSF spectra, drizzle,
// denominator); the iteration then runs as one persistent launch per stage
// over the work units of every field (row tiles, spectral columns, detector
// and target chunks), reusing the single-field kernels' block bodies, so each
// field's arithmetic and summation order are exactly those of its own engine
// (updc/c_core/updc_core.c:1410-1456 per field).  The loop of n iterations
// is captured as one CUDA graph.
#include <algorithm>
#include <map>

#include "engine.cuh"
#include "fft.cuh"
#include "kernels.cuh"
#include "pointwise.cuh"

namespace updc {
namespace {

constexpr int PERSIST_BLOCKS = 148 * 8;  // resident-block budget of a persistent launch

// Device descriptor of one field.
template <typename T> struct FieldDev {
    FftPlan pm, ph;
    const cx<T> *post;
    int W, H, M, FH, ldh, B, nexp, upd_grid;
    FastDiv bdiv;
    size_t nin, nout;
    T scale, max_sens;
    T *estimate, *den, *correction, *blur, *scatter, *wr;
    cx<T> *rx, *y, *rs, *cr, *khat;
    const ExpDesc<T> *exps;
    ExpStats *stats;
    unsigned long long *err;
    double *part_sum, *red_sum;
    unsigned long long *part_neg, *red_neg;
};

// The block's shared copy of a field plan (uniform across the block).
__device__ __forceinline__ void copy_plan(const FftPlan &g, FftPlan &s) {
    const int *src = reinterpret_cast<const int *>(&g);
    int *dst = reinterpret_cast<int *>(&s);
    for (int i = threadIdx.x; i < (int)(sizeof(FftPlan) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// Row R2C of the estimate (src 0, units {field, y0, 0}) or of the scatter
// planes (src 1, units {field, y0, exposure}).
template <typename T, int NT, int CAP>
__global__ void __launch_bounds__(NT, MinBlocks<NT, CAP, T>::value)
    kb_row_r2c(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units, int nunits, int src) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ FftPlan s_plan;
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        copy_plan(f.pm, s_plan);
        const PlaneLoader<T> ld{src == 0 ? f.estimate : f.scatter, f.W, f.nout};
        const SpecRef out{src == 0 ? f.rx : f.rs, f.ldh, (size_t)(f.M + 1) * f.ldh};
        row_r2c_tile<T, NT, CAP, PlaneLoader<T>, false>(s_plan, f.post, ld, f.W, f.H, f.B, f.bdiv, out, nullptr,
                                                        u.y, u.z, smem_raw);
        __syncthreads();
    }
}

// Row C2R + crop of the forward spectra into the blur planes (src 0, units
// {field, y0, exposure}) or of the adjoint spectrum into the correction
// (src 1, units {field, y0, 0}).
template <typename T, int NT, int CAP>
__global__ void __launch_bounds__(NT, MinBlocks<NT, CAP, T>::value)
    kb_row_c2r(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units, int nunits, int src) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ FftPlan s_plan;
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        copy_plan(f.pm, s_plan);
        const SpecRef in{src == 0 ? f.y : f.cr, f.ldh, (size_t)(f.M + 1) * f.ldh};
        const PlaneStore<T> epi{src == 0 ? f.blur : f.correction, f.W, f.nout};
        row_c2r_tile<T, NT, CAP, PlaneStore<T>, false>(s_plan, f.post, in, nullptr, f.H, f.W, f.B, f.bdiv, f.scale,
                                                       epi, f.err, u.y, u.z, smem_raw);
        __syncthreads();
    }
}

// Column pass of the forward model, units {field, u}.
template <typename T, int NT, int CAP>
__global__ void __launch_bounds__(NT, MinBlocks<NT, CAP, T>::value)
    kb_col_forward(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units, int nunits) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ FftPlan s_plan;
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        copy_plan(f.ph, s_plan);
        const size_t nu = (size_t)f.M + 1;
        col_forward_column<T, NT, CAP>(s_plan, f.rx, f.ldh, f.H, f.khat, nu * f.FH, f.nexp, f.y, f.ldh, nu * f.ldh,
                                       f.H, nullptr, u.y, smem_raw);
        __syncthreads();
    }
}

// Column pass of the adjoint (conj-OTF sum over the field's exposures), units {field, u}.
template <typename T, class Acc, int NT, int CAP>
__global__ void __launch_bounds__(NT, MinBlocks<NT, CAP, T>::value)
    kb_col_adjoint(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units, int nunits) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ FftPlan s_plan;
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        copy_plan(f.ph, s_plan);
        const size_t nu = (size_t)f.M + 1;
        col_adjoint_column<T, Acc, NT, CAP>(s_plan, f.rs, f.ldh, nu * f.ldh, f.H, f.khat, nu * f.FH, f.nexp, f.cr,
                                            f.ldh, f.H, nullptr, u.y, smem_raw);
        __syncthreads();
    }
}

// Detector loop, units {field, exposure, block, blocks of the exposure}.
template <typename T, bool COMP>
__global__ void __launch_bounds__(DET_WARPS * 32)
    kb_detector(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units, int nunits) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        const ExpDesc<T> e = f.exps[u.y];
        detector_tiles<T, COMP>(e, u.y, f.nin, f.blur + (size_t)u.y * f.nout, f.wr + (size_t)u.y * f.nin, f.stats,
                                f.err, (unsigned)u.z, (unsigned)u.w, smem_raw);
        __syncthreads();
    }
}

// Transposed gather S^T (W ratio), units {field, exposure, block, blocks}.
template <typename T>
__global__ void __launch_bounds__(256) kb_scatter(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units,
                                                  int nunits) {
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        const ExpDesc<T> e = f.exps[u.y];
        scatter_targets<T, T, T>(e, f.nout, f.wr + (size_t)u.y * f.nin, 0, f.scatter + (size_t)u.y * f.nout,
                                 (unsigned)u.z, (unsigned)u.w);
    }
}

// Multiplicative update, units {field, block} with each field's own grid.
template <typename T>
__global__ void __launch_bounds__(256) kb_update(const FieldDev<T> *__restrict__ F, const int4 *__restrict__ units,
                                                 int nunits) {
    for (int i = blockIdx.x; i < nunits; i += gridDim.x) {
        const int4 u = units[i];
        const FieldDev<T> &f = F[u.x];
        update_block_vec<T>(f.nout, f.correction, f.den, f.estimate, f.max_sens, f.err, f.part_sum, f.part_neg,
                            (unsigned)u.y, (unsigned)f.upd_grid);
        __syncthreads();
    }
}

// One block per field: partial sums -> signed sum, negative count.
template <typename T> __global__ void __launch_bounds__(256) kb_reduce(const FieldDev<T> *__restrict__ F) {
    const FieldDev<T> &f = F[blockIdx.x];
    reduce_partials_block(f.part_sum, f.part_neg, f.upd_grid, f.red_sum, f.red_neg);
}

// Per-iteration reset of every field's FreezeMu counters and error record.
template <typename T> __global__ void kb_reset(const FieldDev<T> *__restrict__ F) {
    const FieldDev<T> &f = F[blockIdx.x];
    for (int k = threadIdx.x; k < f.nexp; k += blockDim.x) f.stats[k] = ExpStats{0, 0, ~0ull, 0};
    if (threadIdx.x == 0) *f.err = ~0ull;
}

// Record of field blockIdx.x for one iteration: {err, signed sum, negative,
// then per exposure nnew, ntotal} at rec + offset[field] (8-byte words).
template <typename T>
__global__ void kb_records(const FieldDev<T> *__restrict__ F, const int *__restrict__ offset,
                           unsigned long long *__restrict__ rec) {
    const FieldDev<T> &f = F[blockIdx.x];
    unsigned long long *r = rec + offset[blockIdx.x];
    if (threadIdx.x == 0) {
        r[0] = *f.err;
        r[1] = (unsigned long long)__double_as_longlong(*f.red_sum);
        r[2] = *f.red_neg;
    }
    for (int k = threadIdx.x; k < f.nexp; k += blockDim.x) {
        r[3 + 2 * k] = f.stats[k].nnew;
        r[4 + 2 * k] = f.stats[k].ntotal;
    }
}

template <typename T> class BatchImpl final : public Batch {
  public:
    explicit BatchImpl(const EngineOptions &opt) : opt_(opt) {
        opt_.use_graph = 0;
        opt_.stage_timing = 0;
        UPDC_CUDA(cudaSetDevice(opt_.device));
        UPDC_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    }
    ~BatchImpl() override {
        drop_graphs();
        for (void *p : allocs_) cudaFree(p);
        if (pinned_) cudaFreeHost(pinned_);
        for (auto e : events_) cudaEventDestroy(e);
        fields_.clear();
        if (stream_) cudaStreamDestroy(stream_);
    }

    void add_field(const std::string &manifest, int W, int H, int iw, int ih, int nexp, int transposed) override {
        if (setup_done_) throw Error(1, "fields are added before setup");
        auto e = make_engine(opt_);
        e->load(manifest, W, H, iw, ih, nexp, transposed);
        fields_.push_back(std::move(e));
    }
    int fields() const override { return (int)fields_.size(); }
    Engine &field(int i) override { return *fields_.at(i); }
    size_t units(int stage) const override { return stage >= 0 && stage < NSTAGE ? nunits_[stage] : 0; }

    void setup() override {
        if (fields_.empty()) throw Error(1, "the batch has no field");
        std::vector<FieldDev<T>> h;
        for (size_t i = 0; i < fields_.size(); ++i) {
            fields_[i]->setup();
            const FieldView v = fields_[i]->field_view();
            if (v.elem_bytes != (int)sizeof(T)) throw Error(1, "field precision differs from the batch");
            if (v.needs_aux)
                throw Error(1, "field " + std::to_string(i) + ": FFT height too large for a batched column transform");
            FieldDev<T> d{};
            d.pm = v.plan_m, d.ph = v.plan_h;
            d.post = (const cx<T> *)v.post;
            d.W = v.W, d.H = v.H, d.M = v.M, d.FH = v.FH, d.ldh = v.ldh, d.B = v.row_b, d.nexp = v.nexp;
            d.upd_grid = v.upd_grid;
            d.bdiv = FastDiv((uint32_t)v.row_b);
            d.nin = v.nin, d.nout = v.nout;
            d.scale = (T)v.scale, d.max_sens = (T)v.max_sens;
            d.estimate = (T *)v.estimate, d.den = (T *)v.den, d.correction = (T *)v.correction;
            d.blur = (T *)v.blur, d.scatter = (T *)v.scatter, d.wr = (T *)v.wr;
            d.rx = (cx<T> *)v.rx, d.y = (cx<T> *)v.y, d.rs = (cx<T> *)v.rs, d.cr = (cx<T> *)v.cr;
            d.khat = (cx<T> *)v.khat;
            d.exps = (const ExpDesc<T> *)v.exps;
            d.stats = (ExpStats *)v.stats;
            d.err = v.err;
            d.part_sum = v.part_sum, d.red_sum = v.red_sum, d.part_neg = v.part_neg, d.red_neg = v.red_neg;
            h.push_back(d);
            comp_mu_ = v.comp_mu;
            smem_row_ = std::max(smem_row_, row_buf_bytes(v.row_b, v.M, sizeof(cx<T>), v.plan_m.pad_shift));
            const size_t fb = fft_buf_bytes(v.FH, sizeof(cx<T>), v.plan_h.pad_shift);
            smem_fwd_ = std::max(smem_fwd_, fb + align16((size_t)v.FH * sizeof(cx<T>)));
            smem_adj_ = std::max(smem_adj_, fb + align16((size_t)v.FH * acc_bytes()));
        }
        host_ = h;
        d_fields_ = alloc<FieldDev<T>>(h.size());
        UPDC_CUDA(cudaMemcpy(d_fields_, h.data(), h.size() * sizeof(FieldDev<T>), cudaMemcpyHostToDevice));
        build_units();
        if (smem_row_ > SPEC_SMEM_LIMIT || smem_fwd_ > SPEC_SMEM_LIMIT || smem_adj_ > SPEC_SMEM_LIMIT)
            throw Error(1, "batched transforms exceed the shared-memory limit");
        set_attr(kb_detector<T, true>, sizeof(DetShared));
        set_attr(kb_detector<T, false>, sizeof(DetShared));
        set_attr(kb_row_r2c<T, SpecRowNt<T>::value, SpecCaps<T>::ROW>, smem_row_);
        set_attr(kb_row_c2r<T, SpecRowNt<T>::value, SpecCaps<T>::ROW>, smem_row_);
        set_attr(kb_col_forward<T, SPEC_NT, SpecCaps<T>::COL_S>, smem_fwd_);
        if constexpr (sizeof(T) == 4) {
            set_attr(kb_col_adjoint<T, AccF64, SpecNtAdj<T>::value, SpecCaps<T>::COL_S>, smem_adj_);
            set_attr(kb_col_adjoint<T, AccKahan, SpecNtAdj<T>::value, SpecCaps<T>::COL_S>, smem_adj_);
        }
        set_attr(kb_col_adjoint<T, AccPlain<T>, SpecNtAdj<T>::value, SpecCaps<T>::COL_S>, smem_adj_);
        // record layout: per field {err, sum, negative, 2 words per exposure}
        std::vector<int> off(h.size());
        rec_words_ = 0;
        for (size_t i = 0; i < h.size(); ++i) {
            off[i] = rec_words_;
            rec_words_ += 3 + 2 * h[i].nexp;
        }
        d_rec_offset_ = alloc<int>(off.size());
        UPDC_CUDA(cudaMemcpy(d_rec_offset_, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
        rec_offset_ = off;
        UPDC_CUDA(cudaDeviceSynchronize());
        setup_done_ = true;
    }

    void iterate(int n, bool check_each, std::vector<BatchRecord> *records) override {
        if (!setup_done_) throw Error(1, "batch is not set up");
        if (n < 1) return;
        ensure_records(n);
        while ((int)events_.size() < 2 * n) {
            cudaEvent_t e;
            UPDC_CUDA(cudaEventCreate(&e));
            events_.push_back(e);
        }
        int done = 0;
        while (done < n) {
            const int batch = check_each ? 1 : std::min(n - done, LOOP_GRAPH_MAX);
            if (batch > 1) {
                UPDC_CUDA(cudaGraphLaunch(loop_graph(batch), stream_));
            } else {
                enqueue_recorded(0, false);
            }
            UPDC_CUDA(cudaMemcpyAsync(pinned_, d_rec_, (size_t)batch * rec_words_ * 8, cudaMemcpyDeviceToHost, stream_));
            UPDC_CUDA(cudaStreamSynchronize(stream_));
            parse(batch, records);
            done += batch;
        }
    }

  private:
    static constexpr int NSTAGE = 8;  // est rows, columns, forward rows, detector, scatter, scatter rows, update, adjoint rows
    static constexpr int LOOP_GRAPH_MAX = 64;
    EngineOptions opt_;
    std::vector<std::unique_ptr<Engine>> fields_;
    std::vector<FieldDev<T>> host_;
    FieldDev<T> *d_fields_ = nullptr;
    int4 *d_units_[NSTAGE] = {};
    size_t nunits_[NSTAGE] = {};
    size_t smem_row_ = 0, smem_fwd_ = 0, smem_adj_ = 0;
    int comp_mu_ = 0;
    bool setup_done_ = false;
    cudaStream_t stream_ = nullptr;
    std::vector<void *> allocs_;
    std::vector<cudaEvent_t> events_;
    std::map<int, cudaGraphExec_t> graphs_;
    int rec_words_ = 0;
    std::vector<int> rec_offset_;
    int *d_rec_offset_ = nullptr;
    unsigned long long *d_rec_ = nullptr;
    void *pinned_ = nullptr;
    int rec_capacity_ = 0;

    template <typename U> U *alloc(size_t n) {
        U *p = nullptr;
        UPDC_CUDA(cudaMalloc(&p, (n ? n : 1) * sizeof(U)));
        allocs_.push_back(p);
        return p;
    }
    template <typename K> static void set_attr(K kern, size_t bytes) {
        raise_smem_limit(reinterpret_cast<const void *>(kern), bytes);
    }
    static size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }
    size_t acc_bytes() const {
        if (sizeof(T) == 4 && opt_.form == FORM_FP32) return sizeof(AccF64::S);
        if (sizeof(T) == 4 && opt_.form == FORM_FP32_KAHAN) return sizeof(AccKahan::S);
        return sizeof(cx<T>);
    }

    // Work units of every stage, largest fields first (their units start
    // first, which evens out the tail of a persistent launch).
    void build_units() {
        std::vector<int> order(host_.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return (size_t)host_[a].FH * (host_[a].M + 1) > (size_t)host_[b].FH * (host_[b].M + 1);
        });
        std::vector<int4> u[NSTAGE];
        for (int f : order) {
            const FieldDev<T> &d = host_[f];
            for (int y0 = 0; y0 < d.H; y0 += d.B) {
                u[0].push_back(make_int4(f, y0, 0, 0));
                u[7].push_back(make_int4(f, y0, 0, 0));
                for (int k = 0; k < d.nexp; ++k) {
                    u[2].push_back(make_int4(f, y0, k, 0));
                    u[5].push_back(make_int4(f, y0, k, 0));
                }
            }
            for (int c = 0; c <= d.M; ++c) u[1].push_back(make_int4(f, c, 0, 0));
            const int nbd = (int)std::min<size_t>(ceil_div(d.nin, 256), PERSIST_BLOCKS);
            const int nbs = (int)std::min<size_t>(ceil_div(d.nout, 256), PERSIST_BLOCKS);
            for (int k = 0; k < d.nexp; ++k) {
                for (int b = 0; b < nbd; ++b) u[3].push_back(make_int4(f, k, b, nbd));
                for (int b = 0; b < nbs; ++b) u[4].push_back(make_int4(f, k, b, nbs));
            }
            for (int b = 0; b < d.upd_grid; ++b) u[6].push_back(make_int4(f, b, 0, 0));
        }
        for (int s = 0; s < NSTAGE; ++s) {
            nunits_[s] = u[s].size();
            d_units_[s] = alloc<int4>(u[s].size());
            UPDC_CUDA(cudaMemcpy(d_units_[s], u[s].data(), u[s].size() * sizeof(int4), cudaMemcpyHostToDevice));
        }
    }
    static unsigned grid_for(size_t units) { return (unsigned)std::max<size_t>(1, std::min<size_t>(units, PERSIST_BLOCKS)); }

    void enqueue_iteration() {
        const int nf = (int)host_.size();
        constexpr int NT = SPEC_NT, RNT = SpecRowNt<T>::value;
        constexpr int ROW = SpecCaps<T>::ROW, COL = SpecCaps<T>::COL_S;
        kb_reset<T><<<nf, 32, 0, stream_>>>(d_fields_);
        kb_row_r2c<T, RNT, ROW><<<grid_for(nunits_[0]), RNT, smem_row_, stream_>>>(d_fields_, d_units_[0], (int)nunits_[0], 0);
        kb_col_forward<T, NT, COL><<<grid_for(nunits_[1]), NT, smem_fwd_, stream_>>>(d_fields_, d_units_[1], (int)nunits_[1]);
        kb_row_c2r<T, RNT, ROW><<<grid_for(nunits_[2]), RNT, smem_row_, stream_>>>(d_fields_, d_units_[2], (int)nunits_[2], 0);
        if (comp_mu_)
            kb_detector<T, true><<<grid_for(nunits_[3]), DET_WARPS * 32, sizeof(DetShared), stream_>>>(d_fields_, d_units_[3], (int)nunits_[3]);
        else
            kb_detector<T, false><<<grid_for(nunits_[3]), DET_WARPS * 32, sizeof(DetShared), stream_>>>(d_fields_, d_units_[3], (int)nunits_[3]);
        kb_scatter<T><<<grid_for(nunits_[4]), 256, 0, stream_>>>(d_fields_, d_units_[4], (int)nunits_[4]);
        kb_row_r2c<T, RNT, ROW><<<grid_for(nunits_[5]), RNT, smem_row_, stream_>>>(d_fields_, d_units_[5], (int)nunits_[5], 1);
        launch_adjoint();
        kb_row_c2r<T, RNT, ROW><<<grid_for(nunits_[7]), RNT, smem_row_, stream_>>>(d_fields_, d_units_[7], (int)nunits_[7], 1);
        kb_update<T><<<grid_for(nunits_[6]), 256, 0, stream_>>>(d_fields_, d_units_[6], (int)nunits_[6]);
        kb_reduce<T><<<nf, 256, 0, stream_>>>(d_fields_);
        UPDC_CUDA(cudaGetLastError());
    }
    void launch_adjoint() {
        constexpr int NTA = SpecNtAdj<T>::value, COL = SpecCaps<T>::COL_S;
        const unsigned g = grid_for(nunits_[1]);
        if constexpr (sizeof(T) == 4) {
            if (opt_.form == FORM_FP32) {
                kb_col_adjoint<T, AccF64, NTA, COL><<<g, NTA, smem_adj_, stream_>>>(d_fields_, d_units_[1], (int)nunits_[1]);
                return;
            }
            if (opt_.form == FORM_FP32_KAHAN) {
                kb_col_adjoint<T, AccKahan, NTA, COL><<<g, NTA, smem_adj_, stream_>>>(d_fields_, d_units_[1], (int)nunits_[1]);
                return;
            }
        }
        kb_col_adjoint<T, AccPlain<T>, NTA, COL><<<g, NTA, smem_adj_, stream_>>>(d_fields_, d_units_[1], (int)nunits_[1]);
    }

    // One iteration with its events (external record nodes inside a
    // capture) and its record written to slot i of the device record buffer.
    void enqueue_recorded(int i, bool capturing) {
        const unsigned flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
        UPDC_CUDA(cudaEventRecordWithFlags(events_[2 * i], stream_, flags));
        enqueue_iteration();
        UPDC_CUDA(cudaEventRecordWithFlags(events_[2 * i + 1], stream_, flags));
        kb_records<T><<<(unsigned)host_.size(), 32, 0, stream_>>>(d_fields_, d_rec_offset_, d_rec_ + (size_t)i * rec_words_);
        UPDC_CUDA(cudaGetLastError());
    }
    void drop_graphs() {
        for (auto &g : graphs_) cudaGraphExecDestroy(g.second);
        graphs_.clear();
    }
    cudaGraphExec_t loop_graph(int n) {
        auto it = graphs_.find(n);
        if (it != graphs_.end()) return it->second;
        if (graphs_.size() >= 8) drop_graphs();
        cudaGraph_t g = nullptr;
        UPDC_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            for (int i = 0; i < n; ++i) enqueue_recorded(i, true);
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
        graphs_[n] = ex;
        return ex;
    }
    void ensure_records(int n) {
        const int need = std::min(n, LOOP_GRAPH_MAX);
        if (need <= rec_capacity_) return;
        drop_graphs();  // they write into the old buffer
        d_rec_ = alloc<unsigned long long>((size_t)need * rec_words_);
        if (pinned_) cudaFreeHost(pinned_);
        UPDC_CUDA(cudaMallocHost(&pinned_, (size_t)need * rec_words_ * 8));
        rec_capacity_ = need;
    }
    void parse(int batch, std::vector<BatchRecord> *records) {
        const unsigned long long *src = (const unsigned long long *)pinned_;
        for (int i = 0; i < batch; ++i) {
            const unsigned long long *r = src + (size_t)i * rec_words_;
            for (size_t f = 0; f < host_.size(); ++f) {
                const unsigned long long key = r[rec_offset_[f]];
                if (key != ~0ull)
                    throw Error(1, "field " + std::to_string(f) + ": " + error_message((uint32_t)(key & 0xFF)));
            }
            if (!records) continue;
            BatchRecord rec;
            float ms = 0;
            UPDC_CUDA(cudaEventElapsedTime(&ms, events_[2 * i], events_[2 * i + 1]));
            rec.seconds = ms * 1e-3;
            for (size_t f = 0; f < host_.size(); ++f) {
                const unsigned long long *q = r + rec_offset_[f];
                double s;
                memcpy(&s, &q[1], 8);
                rec.signed_sum.push_back(s);
                rec.negative.push_back(q[2]);
                for (int k = 0; k < host_[f].nexp; ++k) {
                    rec.new_frozen.push_back(q[3 + 2 * k]);
                    rec.total_frozen.push_back(q[4 + 2 * k]);
                }
            }
            records->push_back(std::move(rec));
        }
    }
};

}  // namespace

std::unique_ptr<Batch> make_batch(const EngineOptions &opt) {
    if (opt.form == FORM_FP64) return std::unique_ptr<Batch>(new BatchImpl<double>(opt));
    return std::unique_ptr<Batch>(new BatchImpl<float>(opt));
}

}  // namespace updc
