// cufsp_sparse.cu -- sparse-format generator for non-factorisable propensities.
//
// Stands in for the reference's CUDA_CSR and HYB formats (src/fspmat_csr_kernels.cu,
// src/fspmat_hyb_kernels.cu).  Every row of every per-reaction matrix A_r has the diagonal
// -a_r(x_i) and at most one off-diagonal a_r(x_i - nu_r) at column i - d_r, so instead of
// storing values AND column indices (HYB: 20 B per state and reaction) the build stores the
// propensity table P[r][i] = a_r(x_i) once (8 B per state and reaction):
//   diag  = -P[r][i]
//   off   =  P[r][i - d_r]   when x_i - nu_r lies in the box (tested on the decoded state)
// The action streams P[.][i] and gathers P[r][i - d_r] and x[i - d_r] through L2.
//
// The table is filled on the device by calling the propensity for every (state, reaction):
// a device function pointer (the reference's PropFun, src/cme_util.h:25, called exactly as
// fspmat_hyb_fill_data does at src/fspmat_hyb_kernels.cu:44-53) or the product of factor
// tables, multiplied in species order ((1 * f_0) * f_1) * ...
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "cufsp_internal.h"
#define CUFSP_SPARSE_RTC_MAX_R 64
#include "cufsp_sparse_rtc.cuh"

namespace cufsp {

namespace {
const char *kSparseSource =
#include "cufsp_sparse_src.inc"
    ;
}  // namespace

struct SparseArgs {
    const double *__restrict__ P;       // [nr][n]
    const int *__restrict__ rinfo;      // [nr][2 + ns]: d_r, touched-species mask, nu_{r,0..ns-1}
    const double *__restrict__ d_alpha; // nullable
    const int *__restrict__ d_skip;     // nullable: return at once when *d_skip != 0
    int64_t n;
    int ns, nr;
    int i_begin, i_end;
    FastDiv div[CUFSP_MAX_SPECIES];
    int bnd[CUFSP_MAX_SPECIES];
    double coef[CUFSP_MAX_REACTIONS_SPARSE];
};

template <int NSB>
__device__ __forceinline__ void decode_state(uint32_t i, const FastDiv *div, int ns, int (&xs)[NSB]) {
#pragma unroll
    for (int s = 0; s < NSB; ++s) {
        if (s < ns) {
            const uint32_t q = fd_div(i, div[s]);
            xs[s] = (int)(i - q * div[s].d);
            i = q;
        } else {
            xs[s] = 0;
        }
    }
}

template <int NSB, bool ACCUM>
__global__ void __launch_bounds__(256) k_sparse_mv(const SparseArgs a, const double *__restrict__ x,
                                                   double *__restrict__ y) {
    extern __shared__ int s_rinfo[];
    if (a.d_skip && *a.d_skip) return;
    const int w = 2 + a.ns;
    for (int t = threadIdx.x; t < a.nr * w; t += blockDim.x) s_rinfo[t] = __ldg(a.rinfo + t);
    __syncthreads();
    const double alpha_dev = a.d_alpha ? __ldg(a.d_alpha) : 1.0;
    const int64_t nm1 = a.n - 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = a.i_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.i_end; i += stride) {
        int xs[NSB];
        decode_state<NSB>((uint32_t)i, a.div, a.ns, xs);
        const double xi = __ldg(x + i);
        double diag = 0.0, off = 0.0;
#pragma unroll 4
        for (int r = 0; r < a.nr; ++r) {
            const int *ri = s_rinfo + r * w;
            const int d = ri[0];
            const unsigned mask = (unsigned)ri[1];
            bool ok = true;
#pragma unroll
            for (int s = 0; s < NSB; ++s) {
                if ((mask >> s) & 1u) {
                    const int xsh = xs[s] - ri[2 + s];
                    ok = ok && xsh >= 0 && xsh <= a.bnd[s];
                }
            }
            int64_t src = i - d;
            src = src < 0 ? 0 : (src > nm1 ? nm1 : src);
            const double *Pr = a.P + (size_t)r * a.n;
            const double c = a.coef[r];
            diag = fma(c, __ldcs(Pr + i), diag);
            const double pv = __ldg(Pr + src) * __ldg(x + src);
            off = fma(c, ok ? pv : 0.0, off);
        }
        double out = alpha_dev * fma(-diag, xi, off);
        if (ACCUM) out += y[i];
        y[i] = out;
    }
}

struct FillArgs {
    const double *__restrict__ tables;
    cufsp_prop_fn prop;
    int64_t n;
    int ns, nr, tab_stride;
    FastDiv div[CUFSP_MAX_SPECIES];
    int tab_off[CUFSP_MAX_SPECIES];
};

__global__ void __launch_bounds__(256) k_sparse_fill(const FillArgs a, double *__restrict__ P) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        int xs[CUFSP_MAX_SPECIES];
        uint32_t rem = (uint32_t)i;
        for (int s = 0; s < a.ns; ++s) {
            const uint32_t q = fd_div(rem, a.div[s]);
            xs[s] = (int)(rem - q * a.div[s].d);
            rem = q;
        }
        for (int r = 0; r < a.nr; ++r) {
            double v;
            if (a.prop) {
                v = a.prop(xs, r);
            } else {
                const double *t = a.tables + (size_t)r * a.tab_stride;
                v = 1.0;
                for (int s = 0; s < a.ns; ++s) v *= __ldg(t + a.tab_off[s] + xs[s]);
            }
            P[(size_t)r * a.n + i] = v;
        }
    }
}

struct SparseData {
    int64_t n = 0;
    int ns = 0, nr = 0;
    double *d_P = nullptr;
    int *d_rinfo = nullptr;
    std::vector<int> bounds;
    int64_t halo = 0;
    int grid_full = 0;
    // kernel specialised for this network and box (cufsp_sparse_rtc.cuh); null: k_sparse_mv
    std::shared_ptr<RtcModule> rtc;
    int rtc_grid = 0;
    std::string describe;
};

namespace {

// Compiles the specialised kernel for this network and box; sets sd->rtc or the reason in `why`.
void sparse_build_rtc(const ModelHost &m, SparseData *sd, std::string &why) {
    const char *ev = getenv("CUFSP_SPARSE_RTC");
    if (ev && atoi(ev) == 0) {
        why = "disabled (CUFSP_SPARSE_RTC=0)";
        return;
    }
    if (m.nr > CUFSP_SPARSE_RTC_MAX_R) {
        why = "more than 64 reactions";
        return;
    }
    if (m.n % 2 != 0) {  // table rows of 16-byte pairs need an even row length
        why = "odd number of states";
        return;
    }
    std::vector<int64_t> stride(m.ns);
    int64_t st = 1;
    for (int s = 0; s < m.ns; ++s) {
        stride[s] = st;
        st *= (int64_t)m.bounds[s] + 1;
    }
    // Reactions whose loads are in flight together, and CTAs per SM the launch bounds promise
    // (CUFSP_SPARSE_CHUNK / CUFSP_SPARSE_MINB override them for tuning).  Measured on the 255^3
    // 9-reaction workload (B200): chunks of 5 at 2 CTAs per SM 275 us per action (5.86 TB/s), all 9
    // at once 331 us, the generic kernel 748 us.
    const char *ec = getenv("CUFSP_SPARSE_CHUNK");
    const char *em = getenv("CUFSP_SPARSE_MINB");
    const int chunk = std::max(1, std::min(m.nr, ec ? atoi(ec) : 5));
    const int minb = std::max(1, std::min(8, em ? atoi(em) : 2));
    std::ostringstream o;
    o << "#define CUFSP_SPARSE_MINB " << minb << "\n";
    o << "#define CUFSP_SPARSE_RTC_MAX_R " << CUFSP_SPARSE_RTC_MAX_R << "\n#define CUFSP_SPARSE_NS " << m.ns
      << "\n#define CUFSP_SPARSE_NR " << m.nr << "\n#define CUFSP_SPARSE_N " << m.n << "LL\n#define CUFSP_SPARSE_CHUNK "
      << chunk << "\nnamespace cufsp_sparse {\n";
    o << "__device__ __forceinline__ constexpr int ext(int s) {";
    for (int s = 0; s < m.ns; ++s) o << " if (s == " << s << ") return " << m.bounds[s] + 1 << ";";
    o << " return 1; }\n";
    o << "__device__ __forceinline__ constexpr int nu(int r, int s) {";
    for (int r = 0; r < m.nr; ++r)
        for (int s = 0; s < m.ns; ++s) {
            const int v = m.nu[(size_t)r * m.ns + s];
            if (v != 0) o << " if (r == " << r << " && s == " << s << ") return " << v << ";";
        }
    o << " return 0; }\n";
    o << "__device__ __forceinline__ constexpr bool touches(int r, int s) { return nu(r, s) != 0; }\n";
    o << "__device__ __forceinline__ constexpr long long shift(int r) {";
    for (int r = 0; r < m.nr; ++r) {
        int64_t d = 0;
        for (int s = 0; s < m.ns; ++s) d += (int64_t)m.nu[(size_t)r * m.ns + s] * stride[s];
        o << " if (r == " << r << ") return " << d << "LL;";
    }
    o << " return 0; }\n}\n";
    sd->rtc = rtc_module(o.str() + kSparseSource, {"cufsp_sparse_mv_accum", "cufsp_sparse_mv_set"}, why);
    if (!sd->rtc) return;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void *)sd->rtc->kernels[0], 256, 0) != cudaSuccess ||
        occ < 1) {
        cudaGetLastError();
        sd->rtc.reset();
        why = "specialised kernel does not fit an SM";
        return;
    }
    sd->rtc_grid = device_info().sm_count * occ;
}

}  // namespace

cufsp_status sparse_create(const ModelHost &m, SparseData **out) {
    SparseData *sd = new SparseData();
    sd->n = m.n;
    sd->ns = m.ns;
    sd->nr = m.nr;
    sd->bounds = m.bounds;
    std::vector<int64_t> stride(m.ns);
    int64_t st = 1;
    for (int s = 0; s < m.ns; ++s) {
        stride[s] = st;
        st *= (int64_t)m.bounds[s] + 1;
    }
    const int w = 2 + m.ns;
    std::vector<int> rinfo((size_t)m.nr * w, 0);
    for (int r = 0; r < m.nr; ++r) {
        int64_t d = 0;
        unsigned mask = 0;
        for (int s = 0; s < m.ns; ++s) {
            const int nu = m.nu[(size_t)r * m.ns + s];
            d += (int64_t)nu * stride[s];
            if (nu != 0) mask |= 1u << s;
            rinfo[(size_t)r * w + 2 + s] = nu;
        }
        if (d > m.n || d < -m.n) d = 0;  // neighbour can never be inside the box; mask test rejects it
        rinfo[(size_t)r * w] = (int)d;
        rinfo[(size_t)r * w + 1] = (int)mask;
        sd->halo = std::max<int64_t>(sd->halo, d < 0 ? -d : d);
    }
    const DeviceInfo &di = device_info();
    sd->grid_full = di.sm_count * 8;
    cudaError_t e = dev_malloc(&sd->d_P, sizeof(double) * (size_t)m.nr * (size_t)m.n);
    if (e == cudaSuccess) e = dev_malloc(&sd->d_rinfo, sizeof(int) * rinfo.size());
    if (e == cudaSuccess) e = cudaMemcpy(sd->d_rinfo, rinfo.data(), sizeof(int) * rinfo.size(), cudaMemcpyHostToDevice);
    double *d_tables = nullptr;
    if (e == cudaSuccess && !m.prop_table.empty()) {  // table evaluated by the caller on the host
        e = cudaMemcpy(sd->d_P, m.prop_table.data(), sizeof(double) * (size_t)m.nr * (size_t)m.n,
                       cudaMemcpyHostToDevice);
    } else if (e == cudaSuccess && !m.prop_device) {
        e = dev_malloc(&d_tables, sizeof(double) * m.tables.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(d_tables, m.tables.data(), sizeof(double) * m.tables.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && m.prop_table.empty()) {
        FillArgs f;
        f.tables = d_tables;
        f.prop = m.prop_device;
        f.n = m.n;
        f.ns = m.ns;
        f.nr = m.nr;
        f.tab_stride = m.tab_stride;
        for (int s = 0; s < CUFSP_MAX_SPECIES; ++s) {
            f.div[s] = make_fastdiv(s < m.ns ? (uint32_t)m.bounds[s] + 1u : 1u);
            f.tab_off[s] = s < m.ns ? m.tab_off[s] : 0;
        }
        const int grid = stream_grid(m.n, 1, di.sm_count * 8);
        k_sparse_fill<<<grid, 256>>>(f, sd->d_P);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    if (d_tables) cudaFree(d_tables);
    if (e != cudaSuccess) {
        sparse_destroy(sd);
        return cuda_error(e, "sparse_create");
    }
    // P must be finite for the action to be well defined.
    std::string why;
    sparse_build_rtc(m, sd, why);
    if (upload_fence() != cudaSuccess) {
        cudaGetLastError();
        sparse_destroy(sd);
        return set_error(CUFSP_ERR_CUDA, "sparse_create: upload failed");
    }
    sd->describe = sd->rtc ? "sparse: propensity table, kernel specialised for the network and box (NVRTC, sm_100a), " +
                                 std::to_string(sd->rtc_grid) + " CTAs x 256 threads"
                           : "sparse: propensity table, k_sparse_mv (" + why + ")";
    *out = sd;
    return CUFSP_SUCCESS;
}

const std::string &sparse_describe(const SparseData *s) { return s->describe; }

void sparse_destroy(SparseData *s) {
    if (!s) return;
    if (s->d_P) cudaFree(s->d_P);
    if (s->d_rinfo) cudaFree(s->d_rinfo);
    delete s;
}

int64_t sparse_halo(const SparseData *s) { return s->halo; }

using SparseKernel = void (*)(const SparseArgs, const double *, double *);

template <int NSB>
static SparseKernel pick_sparse_acc(bool acc) {
    return acc ? k_sparse_mv<NSB, true> : k_sparse_mv<NSB, false>;
}

cufsp_status sparse_apply(SparseData *sd, const double *coefs, double alpha, const double *d_alpha,
                          const int *d_skip, const double *x, bool accumulate, double *y, cudaStream_t st,
                          int64_t i_begin, int64_t i_end) {
    SparseArgs a;
    a.P = sd->d_P;
    a.rinfo = sd->d_rinfo;
    a.d_alpha = d_alpha;
    a.d_skip = d_skip;
    a.n = sd->n;
    a.ns = sd->ns;
    a.nr = sd->nr;
    if (i_end < 0) i_end = sd->n;
    a.i_begin = (int)i_begin;
    a.i_end = (int)i_end;
    for (int s = 0; s < CUFSP_MAX_SPECIES; ++s) {
        a.div[s] = make_fastdiv(s < sd->ns ? (uint32_t)sd->bounds[s] + 1u : 1u);
        a.bnd[s] = s < sd->ns ? sd->bounds[s] : 0;
    }
    for (int r = 0; r < CUFSP_MAX_REACTIONS_SPARSE; ++r) a.coef[r] = r < sd->nr ? alpha * coefs[r] : 0.0;
    const int64_t cnt = i_end - i_begin;
    if (cnt <= 0) return CUFSP_SUCCESS;
    if (sd->rtc && ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % 16) == 0) {
        CufspSparseRtcArgs r;
        std::memset(&r, 0, sizeof(r));
        r.P = sd->d_P;
        r.d_alpha = d_alpha;
        r.d_skip = d_skip;
        r.i_begin = i_begin;
        r.i_end = i_end;
        for (int k = 0; k < sd->nr; ++k) r.coef[k] = alpha * coefs[k];
        const int64_t pairs = (i_end - (i_begin & ~(int64_t)1) + 1) / 2;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(sd->rtc_grid, (pairs + 255) / 256));
        void *args[] = {&r, (void *)&x, (void *)&y};
        CUFSP_CUDA_TRY(cudaLaunchKernel((const void *)sd->rtc->kernels[accumulate ? 0 : 1], dim3(grid), dim3(256), args,
                                        0, st));
        return CUFSP_SUCCESS;
    }
    const int grid = stream_grid(cnt, 2, sd->grid_full);
    const size_t smem = sizeof(int) * (size_t)sd->nr * (2 + sd->ns);
    SparseKernel k = sd->ns <= 2 ? pick_sparse_acc<2>(accumulate)
                     : sd->ns <= 4 ? pick_sparse_acc<4>(accumulate)
                     : sd->ns <= 8 ? pick_sparse_acc<8>(accumulate)
                                   : pick_sparse_acc<16>(accumulate);
    k<<<grid, 256, smem, st>>>(a, x, y);
    CUFSP_CUDA_TRY(cudaGetLastError());
    return CUFSP_SUCCESS;
}

cufsp_status sparse_export(const SparseData *s, double *d_props, cudaStream_t st) {
    CUFSP_CUDA_TRY(cudaMemcpyAsync(d_props, s->d_P, sizeof(double) * (size_t)s->nr * (size_t)s->n,
                                   cudaMemcpyDeviceToDevice, st));
    return CUFSP_SUCCESS;
}

}  // namespace cufsp
