// Cycle control and data-movement kernels.  Built with -fmad=false: the
// stable-time-step arithmetic reproduces the reference's
// update_minVertex_perMaterial_and_dt (Explicit3D/source/exDyna3D.cpp:663-686)
// and run()'s last-step clamp (:90-97) operation by operation.
#include "ensc_device.cuh"
#include "ensc_kernels.h"

#include <algorithm>
#include <cfloat>

namespace ensc {
namespace {

// Sums n values spaced by `stride` in a fixed order: thread t takes
// t, t+NT, t+2NT, ... left to right, then a fixed shared-memory tree.
__device__ double fixed_sum(const double* a, int n) {
    __shared__ double red[kCtlThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kCtlThreads) s = s + a[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kCtlThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// Same fixed order over n values spaced by `stride`.
__device__ double fixed_sum_strided(const double* a, int n, int stride) {
    __shared__ double red[kCtlThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kCtlThreads) s = s + a[static_cast<int64_t>(i) * stride];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kCtlThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// First half of update_minVertex_perMaterial_and_dt for the next cycle
// (exDyna3D.cpp:663-686) and computeSate's clock advance (:775-780): rotate
// dt_i_1 <- dt_i and advance time, unless the total-time clamp (:682-685)
// could fire, which needs the cycle's minimum element edge first
// (edge_prepass + begin_exact).  Caller has checked done / step end.
__device__ __forceinline__ void cycle_begin(Ctl* ctl) {
    ctl->dts_cur = bits_ord(ctl->dts_next);
    ctl->dts_next = kInfBits;
    ctl->len_min = kInfBits;
    const double dt_prev = ctl->dt_i;
    ctl->dt_prev = dt_prev;
    const double time = ctl->time;
    const double time_prev = time + dt_prev;
    // the new dt is factor * min(edge / c, dts_cur) <= factor * dts_cur
    const double bound = ctl->dts_cur * ctl->factor;
    const double rem = ctl->total_time - time_prev;
    const int exact = (rem > 0.0 && rem < bound) ? 1 : 0;
    ctl->need_exact = exact;
    ctl->dt_final = 0;
    if (!exact) {
        double dt_i_1 = dt_prev;
        if (time + dt_i_1 > ctl->step_end) {
            const double r = ctl->step_end - time;
            dt_i_1 = r;
            ctl->dt_i = r;
            ctl->dt_final = 1;
        }
        ctl->dt_i_1 = dt_i_1;
        double t = time + dt_i_1;
        if (t > ctl->total_time) t = ctl->total_time;
        ctl->time = t;
    }
}

// mode 0: the first half of update_minVertex_perMaterial_and_dt for the
// next cycle: rotate dt_i_1 <- dt_i, advance time (computeSate :775-780) and
// fix dt_i_1 unless the total-time clamp (:682-685) could fire, which needs
// this cycle's minimum element edge first (the edge prepass).
// mode 1: fold the energy partials into the control block and clear the work
// partials, which accumulate over cycles between folds (the host folds
// before it reads energies); 2: fold as the initial kinetic energy.
__global__ void __launch_bounds__(kCtlThreads) k_between(Ctl* ctl, Partials P, int mode) {
    if (mode != 0 && (ctl->energy_pending || mode == 2)) {
        const double ei = fixed_sum(P.elem + 0 * P.n_elem_blocks, P.n_elem_blocks);
        const double eh = fixed_sum(P.elem + 1 * P.n_elem_blocks, P.n_elem_blocks);
        const double ev = fixed_sum(P.elem + 2 * P.n_elem_blocks, P.n_elem_blocks);
        const double kin = fixed_sum(P.node + 0 * P.n_node_blocks, P.n_node_blocks);
        const double wx = fixed_sum(P.node + 1 * P.n_node_blocks, P.n_node_blocks);
        if (threadIdx.x == 0) {
            if (mode == 2) {
                ctl->energy[0] = kin;
                ctl->energy[5] = kin;
            } else {
                ctl->energy[0] = kin;
                ctl->energy[1] += ei;
                ctl->energy[2] += eh;
                ctl->energy[3] += ev;
                ctl->energy[4] += wx;
            }
            ctl->energy_pending = 0;
        }
        for (int i = threadIdx.x; i < 3 * P.n_elem_blocks; i += kCtlThreads) P.elem[i] = 0.0;
        for (int i = threadIdx.x; i < P.n_node_blocks; i += kCtlThreads) P.node[P.n_node_blocks + i] = 0.0;
    }
    if (mode != 0 || threadIdx.x != 0 || ctl->done) return;
    if (ctl->status || !(ctl->time < ctl->step_end) || ctl->cycles_done >= ctl->cycles_target ||
        !(ctl->time < ctl->pause_time)) {
        ctl->done = 1;
        return;
    }
    cycle_begin(ctl);
}

// Rest of update_minVertex_perMaterial_and_dt and run()'s clamp for a cycle
// that needed the exact edge minimum (len_min_bits: that minimum, as
// ordered bits).
__device__ __forceinline__ void begin_exact(Ctl* ctl, unsigned long long len_min_bits) {
    const double time = ctl->time;
    double dt_i_1 = ctl->dt_prev;
    const double time_prev = time + dt_i_1;
    double d = bits_ord(len_min_bits) / ctl->wos;
    d = d < ctl->dts_cur ? d : ctl->dts_cur;
    double dt_i = d * ctl->factor;
    if ((ctl->total_time - time_prev) < dt_i && (ctl->total_time - time_prev) > 0.0) {
        dt_i = ctl->total_time - time_prev;
        dt_i_1 = dt_i;
    }
    if (time + dt_i_1 > ctl->step_end) {
        const double r = ctl->step_end - time;
        dt_i = r;
        dt_i_1 = r;
    }
    ctl->dt_i = dt_i;
    ctl->dt_i_1 = dt_i_1;
    ctl->dt_final = 1;
    double t = time + dt_i_1;
    if (t > ctl->total_time) t = ctl->total_time;
    ctl->time = t;
}

// Minimum element edge over the current coordinates (min_ele_edge,
// exDyna3D.cpp:1173-1220), needed before the element pass only in a cycle
// where the total-time clamp may fire; the last block then applies the clamp
// (begin_exact).
__global__ void __launch_bounds__(128) k_edge_prepass(ElemArrays E, NodeArrays N, Ctl* ctl) {
    if (ctl->done || !ctl->need_exact) return;
    __shared__ unsigned long long red[4];
    const int64_t ep = E.ne_pad, np = N.nn_pad;
    double m = DBL_MAX;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < E.ne;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double xyz[8][3];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t n = E.conn[k * ep + e];
            xyz[k][0] = N.x[n];
            xyz[k][1] = N.x[np + n];
            xyz[k][2] = N.x[2 * np + n];
        }
        constexpr int A0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
        constexpr int A1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
        double mm = DBL_MAX;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const double dx = xyz[A1[k]][0] - xyz[A0[k]][0];
            const double dy = xyz[A1[k]][1] - xyz[A0[k]][1];
            const double dz = xyz[A1[k]][2] - xyz[A0[k]][2];
            const double t = __fma_rn(dz, dz, __fma_rn(dy, dy, dx * dx));  // as the element pass
            mm = t < mm ? t : mm;
        }
        const double len = sqrt(mm);
        m = len < m ? len : m;
    }
    unsigned long long b = ord_bits(m);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, b, o);
        b = w < b ? w : b;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long r = red[0];
        for (int i = 1; i < 4; ++i) r = red[i] < r ? red[i] : r;
        atomicMin(&ctl->len_min, r);
        // the last block to finish takes the edge minimum (through L2: this
        // block may hold an older copy) and begins the cycle (begin_exact)
        __threadfence();
        if (atomicAdd(&ctl->prepass_done, 1) == static_cast<int>(gridDim.x) - 1) {
            __threadfence();
            begin_exact(ctl, atomicOr(&ctl->len_min, 0ull));
            ctl->prepass_done = 0;
        }
    }
}


__global__ void k_arm(Ctl* ctl, double step_end, long long max_cycles, double pause) {
    ctl->step_end = step_end;
    ctl->pause_time = pause;
    ctl->cycles_target = ctl->cycles_done + max_cycles;
    ctl->done = 0;
}

__global__ void k_reset_init(Ctl* ctl) {
    ctl->done = 0;
    ctl->dts_next = kInfBits;
    ctl->len_min = kInfBits;
    ctl->status = 0;
}

// apply_boundary_condition_vec (exDyna3D.cpp:379-490): velocity conditions
// first, fixed DOFs last.
// One velocity component of a node: FP64, or the mixed stepper's float
// (with its residual row, ENSC_MIXED_VLO).
template <typename VT>
__device__ __forceinline__ double load_v(const NodeArrays& N, int c, int64_t n) {
    const int64_t i = c * N.nn_pad + n;
    if constexpr (sizeof(VT) == 4 && ENSC_MIXED_VLO)
        return v_join(static_cast<const float*>(N.v)[i], v_lo_rows(N.v, N.nn_pad)[i]);
    else
        return static_cast<double>(static_cast<const VT*>(N.v)[i]);
}
template <typename VT>
__device__ __forceinline__ void store_v(const NodeArrays& N, int c, int64_t n, double v) {
    const int64_t i = c * N.nn_pad + n;
    if constexpr (sizeof(VT) == 4 && ENSC_MIXED_VLO)
        v_split(v, static_cast<float*>(N.v)[i], v_lo_rows(N.v, N.nn_pad)[i]);
    else
        static_cast<VT*>(N.v)[i] = static_cast<VT>(v);
}

template <typename VT>
__global__ void k_apply_bc_v(NodeArrays N) {
    for (int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; n < N.nn;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const uint32_t code = N.bc[n];
        if (!code) continue;
        for (int c = 0; c < 3; ++c) {
            const uint32_t cc = (code >> (2 * c)) & 3u;
            if (cc & 2u) store_v<VT>(N, c, n, N.bcv[c * N.nn_pad + n]);
            if (cc & 1u) store_v<VT>(N, c, n, 0.0);
        }
    }
}

template <typename VT>
__global__ void __launch_bounds__(kNodeThreads) k_kinetic(NodeArrays N, Partials P) {
    double kin = 0.0;
    for (int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; n < N.nn;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double im = N.inv_mass[n];
        for (int c = 0; c < 3; ++c) {
            const double v = load_v<VT>(N, c, n);
            kin = kin + 0.5 * (v * v) / im;
        }
    }
    __shared__ double red[kNodeThreads];
    red[threadIdx.x] = kin;
    __syncthreads();
    for (int w = kNodeThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        P.node[blockIdx.x] = red[0];
        P.node[P.n_node_blocks + blockIdx.x] = 0.0;
    }
}

// Entry e of the interleaved array is row position at[e] of the SoA rows
// (at null: e).
template <typename ST>
__global__ void k_soa_to_aos(const ST* soa, int64_t n, int64_t pad, int comps, const int32_t* at, double* aos) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n * comps;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = i / comps;
        const int c = static_cast<int>(i - e * comps);
        aos[i] = static_cast<double>(soa[c * pad + (at ? at[e] : e)]);
    }
}

// Displacements of a mixed instance, whose u rows hold the reference
// position xr = x - u: interleaved u = x - xr.
__global__ void k_disp_to_aos(const double* x, const double* xr, int64_t n, int64_t pad, double* aos) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < 3 * n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = i / 3;
        const int64_t k = (i - 3 * e) * pad + e;
        aos[i] = x[k] - xr[k];
    }
}

// a <- x - a over the three node rows: turns the reference position rows of
// a mixed instance into displacement rows and back
__global__ void k_reflect_rows(const double* x, double* a, int64_t n, int64_t pad) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < 3 * n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t c = i / n;
        const int64_t k = c * pad + (i - c * n);
        a[k] = x[k] - a[k];
    }
}

// Velocities between interleaved xyz doubles and the device rows.
template <typename VT>
__global__ void k_v_to_aos(NodeArrays N, double* aos) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < 3 * N.nn;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        aos[i] = load_v<VT>(N, static_cast<int>(i % 3), i / 3);
}
template <typename VT>
__global__ void k_aos_to_v(const double* aos, NodeArrays N) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < 3 * N.nn;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        store_v<VT>(N, static_cast<int>(i % 3), i / 3, aos[i]);
}

template <typename DT>
__global__ void k_aos_to_soa(const double* aos, int64_t n, int64_t pad, int comps, const int32_t* at, DT* soa) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n * comps;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = i / comps;
        const int c = static_cast<int>(i - e * comps);
        soa[c * pad + (at ? at[e] : e)] = static_cast<DT>(aos[i]);
    }
}

// ---- batched instances ---------------------------------------------------------
// Begins every instance's next cycle exactly as k_between does for one
// instance (one thread per instance slot), after marking instances that have
// reached their limits as done, and counts the instances whose cycle needs
// the edge prepass.  The energy terms stay in the per-tile accumulators
// until k_fold_batch.  Each slot's element-pass scalars (dt_i_1, live) go to
// T.sparam; the edge prepass rewrites them where it decides dt.
__global__ void k_begin_batch(BatchTables T, int begin) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= T.counts[2]) return;
    const InstanceDesc& d = T.desc[slot];
    StageHdr h{0.0, 0, 0};
    if (d.active) {
        Ctl* ctl = d.ctl;
        if (!ctl->done) {
            if (ctl->status || !(ctl->time < ctl->step_end) || ctl->cycles_done >= ctl->cycles_target ||
                !(ctl->time < ctl->pause_time)) {
                ctl->done = 1;
            } else if (begin) {
                cycle_begin(ctl);
                if (ctl->need_exact) atomicAdd(T.exact_count, 1);
                h.dt1 = ctl->dt_i_1;
                h.live = 1;
            }
        }
    }
    T.sparam[slot] = h;
}

// Folds an instance's tile accumulators into its control block (one block
// per instance slot, tiles in order): the work terms are added and the tile
// accumulators cleared; the kinetic energy is the sum of the tiles' latest
// values when cycles ran since the last fold.
__global__ void __launch_bounds__(kCtlThreads) k_fold_batch(BatchTables T) {
    const int slot = blockIdx.x;
    if (slot >= T.counts[2]) return;
    const InstanceDesc& d = T.desc[slot];
    if (!d.active) return;
    Ctl* ctl = d.ctl;
    const int nw = T.etile / 32;  // element-tile partials: one per warp
    const int ne_part = d.e_ntiles * nw;
    double* ep = T.etile_part + 3 * static_cast<int64_t>(d.e_tile0) * nw;
    double* np = T.ntile_part + 2 * static_cast<int64_t>(d.n_tile0);
    const double ei = fixed_sum_strided(ep + 0, ne_part, 3);
    const double eh = fixed_sum_strided(ep + 1, ne_part, 3);
    const double ev = fixed_sum_strided(ep + 2, ne_part, 3);
    const double kin = fixed_sum_strided(np + 0, d.n_ntiles, 2);
    const double wx = fixed_sum_strided(np + 1, d.n_ntiles, 2);
    for (int i = threadIdx.x; i < 3 * ne_part; i += kCtlThreads) ep[i] = 0.0;
    for (int i = threadIdx.x; i < d.n_ntiles; i += kCtlThreads) np[2 * i + 1] = 0.0;
    if (threadIdx.x == 0) {
        if (ctl->energy_pending) ctl->energy[0] = kin;
        ctl->energy[1] += ei;
        ctl->energy[2] += eh;
        ctl->energy[3] += ev;
        ctl->energy[4] += wx;
        ctl->energy_pending = 0;
    }
}

// Minimum element edge for the instances whose cycle may hit the total-time
// clamp (see k_edge_prepass), one warp per element tile of T.etile elements.
__global__ void __launch_bounds__(128) k_edge_prepass_batch(BatchTables T) {
    if (*T.exact_count == 0) return;
    const int lane = threadIdx.x & 31;
    const int warp = static_cast<int>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = static_cast<int>((static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5);
    for (int t = warp; t < T.counts[0]; t += nwarps) {
        const InstanceDesc& d = T.desc[T.etile_inst[t]];
        Ctl* ctl = d.ctl;
        if (ctl->done || !ctl->need_exact) continue;
        const int64_t base = T.etile_base[t];
        const int64_t end = base + T.etile < d.E.ne ? base + T.etile : d.E.ne;
        double m = DBL_MAX;
        for (int64_t e = base + lane; e < end; e += 32) {
            const int64_t ep = d.E.ne_pad, np = d.N.nn_pad;
            double xyz[8][3];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t n = d.E.conn[k * ep + e];
                xyz[k][0] = d.N.x[n];
                xyz[k][1] = d.N.x[np + n];
                xyz[k][2] = d.N.x[2 * np + n];
            }
            constexpr int A0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
            constexpr int A1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
            double mm = DBL_MAX;
#pragma unroll
            for (int k = 0; k < 12; ++k) {
                const double dx = xyz[A1[k]][0] - xyz[A0[k]][0];
                const double dy = xyz[A1[k]][1] - xyz[A0[k]][1];
                const double dz = xyz[A1[k]][2] - xyz[A0[k]][2];
                const double tt = __fma_rn(dz, dz, __fma_rn(dy, dy, dx * dx));  // as the element pass
                mm = tt < mm ? tt : mm;
            }
            const double len = sqrt(mm);
            m = len < m ? len : m;
        }
        unsigned long long b = ord_bits(m);
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, b, o);
            b = w < b ? w : b;
        }
        if (lane == 0) atomicMin(&ctl->len_min, b);
    }
    // the last block to finish begins the exact cycles (k_begin_exact for
    // each such instance) and clears the counters
    __shared__ int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(T.prepass_done, 1) == static_cast<int>(gridDim.x) - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int slot = threadIdx.x; slot < T.counts[2]; slot += blockDim.x) {
        const InstanceDesc& d = T.desc[slot];
        if (!d.active) continue;
        Ctl* ctl = d.ctl;
        if (ctl->done || !ctl->need_exact) continue;
        // the edge minimum through L2 (this block may hold an older copy)
        begin_exact(ctl, atomicOr(&ctl->len_min, 0ull));
        T.sparam[slot].dt1 = ctl->dt_i_1;
    }
    if (threadIdx.x == 0) {
        *T.prepass_done = 0;
        *T.exact_count = 0;
    }
}


int grid_for(int64_t work, int threads) {
    const int64_t g = (work + threads - 1) / threads;
    return static_cast<int>(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

}  // namespace

void launch_between_batch(const BatchTables& T, int slots, int mode, cudaStream_t st) {
    if (mode == 1) k_fold_batch<<<slots, kCtlThreads, 0, st>>>(T);
    k_begin_batch<<<(slots + 127) / 128, 128, 0, st>>>(T, mode == 0 ? 1 : 0);
}
void launch_edge_prepass_batch(const BatchTables& T, int grid, cudaStream_t st) {
    k_edge_prepass_batch<<<grid, 128, 0, st>>>(T);
}
void launch_between(Ctl* ctl, const Partials& P, int mode, cudaStream_t st) {
    k_between<<<1, kCtlThreads, 0, st>>>(ctl, P, mode);
}
void launch_edge_prepass(const ElemArrays& E, const NodeArrays& N, Ctl* ctl, int grid, cudaStream_t st) {
    k_edge_prepass<<<grid, 128, 0, st>>>(E, N, ctl);
}
void launch_arm(Ctl* ctl, double step_end, long long max_cycles, cudaStream_t st, double pause) {
    k_arm<<<1, 1, 0, st>>>(ctl, step_end, max_cycles, pause);
}
void launch_reset_init(Ctl* ctl, cudaStream_t st) { k_reset_init<<<1, 1, 0, st>>>(ctl); }
void launch_apply_bc_v(const NodeArrays& N, bool fp32_v, cudaStream_t st) {
    const int g = grid_for(N.nn, 256);
    if (fp32_v) k_apply_bc_v<float><<<g, 256, 0, st>>>(N);
    else k_apply_bc_v<double><<<g, 256, 0, st>>>(N);
}
void launch_kinetic0(const NodeArrays& N, const Partials& P, Ctl* ctl, bool fp32_v, int grid, cudaStream_t st) {
    if (fp32_v) k_kinetic<float><<<grid, kNodeThreads, 0, st>>>(N, P);
    else k_kinetic<double><<<grid, kNodeThreads, 0, st>>>(N, P);
    k_between<<<1, kCtlThreads, 0, st>>>(ctl, P, 2);
}
void launch_soa_to_aos(const void* soa, int64_t n, int64_t pad, int comps, bool src_fp32, double* aos,
                       cudaStream_t st, const int32_t* at) {
    const int g = grid_for(n * comps, 256);
    if (src_fp32) k_soa_to_aos<float><<<g, 256, 0, st>>>(static_cast<const float*>(soa), n, pad, comps, at, aos);
    else k_soa_to_aos<double><<<g, 256, 0, st>>>(static_cast<const double*>(soa), n, pad, comps, at, aos);
}
void launch_disp_to_aos(const double* x, const double* xr, int64_t n, int64_t pad, double* aos, cudaStream_t st) {
    k_disp_to_aos<<<grid_for(3 * n, 256), 256, 0, st>>>(x, xr, n, pad, aos);
}
void launch_reflect_rows(const double* x, double* a, int64_t n, int64_t pad, cudaStream_t st) {
    k_reflect_rows<<<grid_for(3 * n, 256), 256, 0, st>>>(x, a, n, pad);
}
void launch_v_to_aos(const NodeArrays& N, bool fp32_v, double* aos, cudaStream_t st) {
    const int g = static_cast<int>(std::min<int64_t>((3 * N.nn + 255) / 256, 65535));
    if (fp32_v) k_v_to_aos<float><<<g, 256, 0, st>>>(N, aos);
    else k_v_to_aos<double><<<g, 256, 0, st>>>(N, aos);
}
void launch_aos_to_v(const double* aos, const NodeArrays& N, bool fp32_v, cudaStream_t st) {
    const int g = static_cast<int>(std::min<int64_t>((3 * N.nn + 255) / 256, 65535));
    if (fp32_v) k_aos_to_v<float><<<g, 256, 0, st>>>(aos, N);
    else k_aos_to_v<double><<<g, 256, 0, st>>>(aos, N);
}
void launch_aos_to_soa(const double* aos, int64_t n, int64_t pad, int comps, void* soa, bool dst_fp32,
                       cudaStream_t st, const int32_t* at) {
    const int g = grid_for(n * comps, 256);
    if (dst_fp32) k_aos_to_soa<float><<<g, 256, 0, st>>>(aos, n, pad, comps, at, static_cast<float*>(soa));
    else k_aos_to_soa<double><<<g, 256, 0, st>>>(aos, n, pad, comps, at, static_cast<double*>(soa));
}

}  // namespace ensc
