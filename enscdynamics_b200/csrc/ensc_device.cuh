// Device-side data structures shared by the stepper kernels.
//
// Memory layout in HBM (structure of arrays, one array per component so a
// warp of consecutive elements / nodes reads consecutive words):
//   element arrays, length ne (padded stride ne_pad):
//     conn[8][ne_pad] uint32         local node k of element e at conn[k*ne_pad + e]
//     bt[24][ne_pad]                 B0^T row-major per element: (3*k + c)
//     vol0, cbrt_v0, cbrt_v0sq [ne]  per-element constants
//     sigma[6][ne_pad], qia[12][ne_pad], eps_p[ne]
//     fe                             element nodal forces of the current cycle
//                                    (the element -> node hand-off, scratch):
//                                    [24][nn_pad] by node and local slot when
//                                    no node repeats a slot, else [24][ne_pad]
//   node arrays, length nn (stride nn_pad):
//     x[3][nn_pad], u[3][nn_pad] (FP64 always), v[3][nn_pad]
//     inv_mass[nn]                   per node (equal for the 3 DOFs)
//     bc[nn] uint8                   2 bits per DOF (bit0 fixed, bit1 velocity)
//     bcv[3][nn_pad]                 prescribed velocities
//     ell[8][nn_pad] uint32          element holding node n in local slot k, or
//                                    ENSC_NONE; the gather sums slots k = 0..7
//                                    in order, as the reference sums its 8
//                                    slot vectors (exDyna3D.cpp:638-639)
//     csr_ptr/csr_ent                general (slot, element)-sorted lists, used
//                                    instead of ell when a node occupies the
//                                    same slot in more than one element
#pragma once

#include <cmath>
#include <cstring>

#include <cstdint>
#include <cuda_runtime.h>

#define ENSC_NONE 0xFFFFFFFFu

namespace ensc {

// Status bits raised on the device and read back by the host.
enum : int32_t {
    ST_NONFINITE = 1,
    ST_INVERTED = 2,
    ST_BAD_DT = 4,       // stable dt not positive and finite
    ST_TIMEOUT = 8,      // a bounded wait for staged data expired; the pass stopped early
};

// Per-instance control block: the scalar state of exDyna3D's time loop
// (time, dt_i, dt_i_1: exDyna3D.h:175-178) plus the reductions that feed it.
struct Ctl {
    double time, dt_i, dt_i_1;
    double dt_prev;            // dt_i at the start of the cycle
    double step_end, total_time;
    double pause_time;         // stop after the cycle in which time reaches it (no dt clamp)
    double factor, wos;
    double dts_cur;            // min element dt of the previous force pass
    unsigned long long dts_next;   // ordered bits of min element dt, this pass
    unsigned long long len_min;    // ordered bits of min element edge, this pass
    long long cycles_done, cycles_target;
    int32_t done;
    int32_t need_exact;        // total-time clamp possible: edge minimum needed first
    int32_t dt_final;          // dt_i already fixed for this cycle
    int32_t energy_pending;    // partial energy sums of the last cycle not yet folded
    int32_t status;
    int32_t prepass_done;      // blocks of the edge prepass that have finished
    double energy[6];          // kinetic, internal, hourglass, viscous, external, kinetic0
};

// Constants of the mixed-precision element pass, derived once per instance
// on the host (set_mixed_consts).  lambda and 2G are float pairs (hi + lo);
// DRc and CRc are the per-element-invariant factors of the hourglass
// stiffness and damping; the element dt uses 1/wos and cvisq^2/wos in FP64.
struct MixedConsts {
    float G, lam_hi, lam_lo, g2_hi, g2_lo, rho, wos, cvisl, cvisq, y0, H, DRc, CRc, inv_3gh, pad[2];
    double inv_wos, cq2_wos;
};

struct Material {
    double E, nu, rho, G, K, lambda, wos;
    double yield0, hardening;
    double c_dr, c_cr, cvisl, cvisq;
    int32_t plastic;
    int32_t gravity_on;
    double gravity_value, gravity_dir[3];
    // gravity amplitude table: amp_n (time, value) pairs in device memory
    const double* amp;
    int32_t amp_n;
    MixedConsts mc;
};

// Fills M.mc from the FP64 material and controls; call after every change
// of them.
inline void set_mixed_consts(Material& M) {
    MixedConsts& c = M.mc;
    c = MixedConsts{};
    c.G = static_cast<float>(M.G);
    c.lam_hi = static_cast<float>(M.lambda);
    c.lam_lo = static_cast<float>(M.lambda - static_cast<double>(c.lam_hi));
    c.g2_hi = static_cast<float>(2.0 * M.G);
    c.g2_lo = static_cast<float>(2.0 * M.G - static_cast<double>(c.g2_hi));
    c.rho = static_cast<float>(M.rho);
    c.wos = static_cast<float>(M.wos);
    c.cvisl = static_cast<float>(M.cvisl);
    c.cvisq = static_cast<float>(M.cvisq);
    c.y0 = static_cast<float>(M.yield0);
    c.H = static_cast<float>(M.hardening);
    c.DRc = static_cast<float>(M.c_dr * (4.0 / 3.0 * M.G + M.K) * 0.1 / std::sqrt(8.0));
    c.CRc = static_cast<float>(M.c_cr * M.rho * M.wos / 4.0);
    c.inv_3gh = static_cast<float>(1.0 / (3.0 * M.G + M.hardening));
    c.inv_wos = 1.0 / M.wos;
    c.cq2_wos = M.cvisq * M.cvisq / M.wos;
}

struct ElemArrays {
    int64_t ne, ne_pad;
    const uint32_t* conn;
    const void* bt;            // double (FP64) or float (mixed)
    const double* vol0;
    const double* cbrt_v0;
    const double* cbrt_v0sq;
    void* sigma;
    void* qia;
    void* eps_p;
    void* fe;
    // 1 when every element and node array starts 256-byte aligned and
    // ne_pad / nn_pad are multiples of 32: rows of whole 32-entry tiles can be
    // bulk-copied and read as 16-byte vectors (the staged element passes and
    // the vectorised node passes)
    int32_t tiles_aligned;
    // 1: fe is node-major, fe[(3k + c) * nn_pad + conn[k][e]] -- the
    // reference's per-local-slot nodal vectors (exDyna3D.cpp:523-634), each
    // entry written by the one element that holds the node in slot k;
    // 0: fe is element-major, fe[(3k + c) * ne_pad + e], gathered through
    // ell / csr by the node pass
    int32_t slot_major;
};

// Elements per patch of the mixed patch assembly: one staged tile.
constexpr int kPatchElems = 64;

// The tables of the patch assembly (mixed precision), kept apart from the
// element and node arrays so that kernels of the slot assembly see the same
// argument layout either way; all null for an instance on the slot
// assembly.  Elements are stored in patches of kPatchElems consecutive
// elements.  The element pass sums a patch's element forces per patch node
// in shared memory and writes one partial per (patch, node): patch p's
// nodes are the partial entries pf_off[p] .. pf_off[p + 1] - 1, entry q's
// incidences are pinc[pinc_off[q] .. pinc_off[q + 1]) as (element in patch
// << 3 | slot), in slot order, and its partial goes to pf[c * pf_pad + q].
// Node n's force is the sum of its partials nent[nptr[n] .. nptr[n + 1]),
// in patch order.  iperm maps an element of the caller's numbering to its
// stored position.
struct PatchArrays {
    const uint32_t* pf_off;
    const uint32_t* pinc_off;
    const uint16_t* pinc;
    float* pf;
    int64_t pf_pad;
    const uint32_t* nptr;
    const uint32_t* nent;
    const int32_t* iperm;
};

struct NodeArrays {
    int64_t nn, nn_pad;
    double* x;
    double* u;
    void* v;                   // double (FP64) or float (mixed)
    const double* inv_mass;
    const uint8_t* bc;
    const double* bcv;
    const uint32_t* ell;
    const int64_t* csr_ptr;    // non-null: use the general lists
    const uint32_t* csr_ent;   // (e << 3) | slot
    const uint8_t* slot_mask;  // slot-major forces: bit k set if slot k holds an element
    double* rf;                // reactions, [3][nn_pad]
};

// Partial sums written by each block of a pass, folded in fixed block order.
struct Partials {
    double* elem;              // [3][n_elem_blocks]
    double* node;              // [2][n_node_blocks]
    int32_t n_elem_blocks, n_node_blocks;
};

// The node pass's view of one instance: node arrays, slot-major forces,
// gravity and the control block.  `grouped` is 1 when the forces are
// slot-major and the rows tile-aligned, so W consecutive nodes can be read
// and written as vectors, and 2 for the same under the patch assembly.  In
// a batch, two 128-byte lines per slot; the second is read only under the
// patch assembly.
struct alignas(128) NodeView {
    const void* fe;
    void* v;                   // double (FP64) or float (mixed)
    double* u;
    double* x;
    const double* inv_mass;
    const uint8_t* bc;
    const uint8_t* slot_mask;  // bit k: slot k holds an element
    double* rf;
    Ctl* ctl;
    int64_t nn, np;
    double gravity_value, gravity_dir[3];
    int32_t gravity_on;
    int32_t grouped;
    // patch assembly (pf non-null): node n's force is the sum of
    // pf[c * pf_pad + nent[i]] over i in [nptr[n], nptr[n + 1])
    const float* pf;
    const uint32_t* nptr;
    const uint32_t* nent;
    int64_t pf_pad;
};
static_assert(sizeof(NodeView) == 256, "two lines per slot");

__host__ __device__ inline NodeView node_view(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl,
                                              const PatchArrays* pa = nullptr) {
    NodeView v{};
    v.fe = E.fe;
    v.v = N.v;
    v.u = N.u;
    v.x = N.x;
    v.inv_mass = N.inv_mass;
    v.bc = N.bc;
    v.slot_mask = N.slot_mask;
    v.rf = N.rf;
    v.ctl = ctl;
    v.nn = N.nn;
    v.np = N.nn_pad;
    v.gravity_value = M.gravity_value;
    for (int c = 0; c < 3; ++c) v.gravity_dir[c] = M.gravity_dir[c];
    v.gravity_on = M.gravity_on;
    const bool patch = pa && pa->pf;
    v.grouped = (E.slot_major && E.tiles_aligned) ? (patch ? 2 : 1) : 0;
    if (patch) {
        v.pf = pa->pf;
        v.nptr = pa->nptr;
        v.nent = pa->nent;
        v.pf_pad = pa->pf_pad;
    }
    return v;
}

// ---- batched instances ------------------------------------------------------
// Independent solver instances advanced together: each warp-sized tile (32
// elements or 32 nodes) belongs to one instance, so instance parameters,
// clock and reductions are warp-uniform.
constexpr int kTile = 32;

// The scalars of an instance's node pass in the current cycle (stable dt,
// previous dt, gravity amplitude), computed once per instance.
struct alignas(16) NodeParam {
    double dt_i, dt_i_1, amp;
    int32_t live, pad;
};

// The scalars of an instance's element pass in the current cycle (dt_i_1,
// and whether it runs), written per slot at the start of the cycle and
// bulk-copied into the stage of each of its element tiles.
struct StageHdr {
    double dt1;
    int32_t live, pad;
};

// Where the staged batch element passes copy an element tile from: the
// instance's element rows, each pointer already at the tile's first element.
// A tile's record travels with the stage of the tile two visits earlier, so
// the block that copies a tile reads its record from shared memory.
struct alignas(16) ETileSrc {
    const void* conn;
    const void* bt;
    const void* vol0;
    const void* cbrt_v0;
    const void* cbrt_v0sq;
    const void* sigma;
    const void* qia;
    const void* eps_p;
    int32_t ne_pad;   // row stride in elements
    int32_t cnt;      // entries copied per row (tile size, or the rest of the padded rows)
    int32_t slot, base;
};
static_assert(sizeof(ETileSrc) == 80, "tile records are bulk-copied");

// Written into each stage by the thread that fills it: the tile's instance
// slot and first element.
struct TileInfo {
    int32_t slot, base, pad0, pad1;
};

struct alignas(16) InstanceDesc {
    ElemArrays E;
    NodeArrays N;
    Material M;
    Ctl* ctl;
    int32_t e_tile0, e_ntiles;   // range in the element-tile list
    int32_t n_tile0, n_ntiles;   // range in the node-tile list
    int32_t active;
    int32_t patch;               // 1: the patch assembly, tables in pa
    PatchArrays pa;
};

struct BatchTables {
    const InstanceDesc* desc;    // [slots]
    const int32_t* etile_inst;   // [etiles] instance slot of each element tile
    const int32_t* etile_base;   // first element of the tile within its instance
    const int32_t* ntile_inst;   // [ntiles]
    const int32_t* ntile_base;
    const int32_t* counts;       // [0] element tiles, [1] node tiles, [2] slots in use
    // per-tile energy terms: work done since the last fold (internal,
    // hourglass, viscous; external) and the latest kinetic energy
    double* etile_part;          // [etiles][etile / 32][3] internal / hourglass / viscous work per tile warp
    double* ntile_part;          // [ntiles][2] kinetic energy / external work per tile
    int32_t* exact_count;        // instances whose current cycle needs the edge prepass
    int32_t* prepass_done;       // blocks of the edge prepass that have finished
    int32_t* elem_done;          // blocks of the element pass that have finished
    NodeParam* nparam;           // [slots] this cycle's node-pass scalars
    StageHdr* sparam;            // [slots] this cycle's element-pass scalars
    const NodeView* nview;       // [slots]
    const ETileSrc* etile_src;   // [etiles] copy sources of each element tile
    int32_t etile, ntile;        // elements / nodes per tile
};
static_assert(sizeof(InstanceDesc) % 16 == 0, "instance descriptors are bulk-copied");

// Amplitude factor of gravity in a cycle at `time` with step dt, as
// exDyna3D::deal_amp computes it (exDyna3D.cpp:1222-1278), behaviour kept as
// is: the scan stops at the first segment that ends before `time` (factor
// 1); a cycle inside one segment takes the segment's value at mid-cycle; a
// cycle that crosses segment ends takes the mean of the curve over the cycle,
// where the partial last segment's intercept uses the first segment's slope
// (:1257) and time past the last point counts with value 1.  n < 2: 1.
__host__ __device__ inline double gravity_amplitude(const double* amp, int n, double time, double dt) {
    double y = 1.0;
    for (int i = 0; i + 1 < n; ++i) {
        const double x1 = amp[2 * i], y1 = amp[2 * i + 1];
        const double x2 = amp[2 * i + 2], y2 = amp[2 * i + 3];
        if (time > x2) break;
        const double m = (y2 - y1) / (x2 - x1);
        const double c = y1 - m * x1;
        const double x = time + dt / 2.0;
        if ((x + dt / 2.0) < x2) {
            y = m * x + c;
            break;
        }
        const double dt1 = x2 - time;
        const double xm = time + dt1 / 2.0;
        const double ym = m * xm + c;
        const double a1 = ym * dt1;
        double a2 = 0.0;
        for (int j = 2; j + i < n; ++j) {
            const double xj = amp[2 * (i + j)], yj = amp[2 * (i + j) + 1];
            const double xp = amp[2 * (i + j - 1)], yp = amp[2 * (i + j - 1) + 1];
            if ((x + dt / 2.0) > xj) {
                a2 += (xj - xp) * (yj + yp) / 2.0;
            } else {
                const double mj = (yj - yp) / (xj - xp);
                const double cj = yp - m * xp;
                const double yend = mj * (x + dt / 2.0) + cj;
                a2 += (x + dt / 2.0 - xp) * (yp + yend) / 2.0;
                break;
            }
        }
        const double x_end = amp[2 * (n - 1)];
        if (x + dt / 2.0 > x_end) a2 += (x + dt / 2.0 - x_end) * 1.0;
        y = (a1 + a2) / dt;
        break;
    }
    return y;
}

// ---- mixed-precision velocities ---------------------------------------------
// The mixed stepper keeps each velocity component as a float `hi` (what the
// element pass reads) and a 16-bit residual `lo` in units of 2^-16 of hi's
// spacing: v = hi + lo * ulp(hi) / 2^16, about 40 significant bits.  The node
// pass updates v in FP64 and splits it again, so the velocity integration
// does not drop FP32 rounding every cycle.  In memory the residual rows
// follow the three float rows: [3][nn_pad] float, then [3][nn_pad] int16.
#ifndef ENSC_MIXED_VLO
#define ENSC_MIXED_VLO 1
#endif

// The mixed stepper's element pass forms F from the current coordinates and
// never reads the displacement, so it keeps the reference position
// xr = x - u in the u rows instead of u, and the node pass updates x alone:
// u = x - xr is formed where the state is read (ensc_download, snapshots),
// and an upload of x or u sets xr = x - u.  Both are FP64: u = x - xr is
// within a rounding of x's magnitude of the separately accumulated u.
#ifndef ENSC_MIXED_UREF
#define ENSC_MIXED_UREF 1
#endif

// ulp(hi) / 2^16 and its inverse (normal or zero hi; hi's exponent field e
// gives ulp(hi) = 2^(e - 150), with e = 1 for zero and subnormals)
__host__ __device__ inline double vlo_unit(float hi) {
    uint32_t b;
    memcpy(&b, &hi, sizeof b);
    int e = static_cast<int>((b >> 23) & 0xFFu);
    if (e == 0) e = 1;
    const uint64_t d = static_cast<uint64_t>(e - 166 + 1023) << 52;
    double r;
    memcpy(&r, &d, sizeof r);
    return r;
}
__host__ __device__ inline double vlo_inv_unit(float hi) {
    uint32_t b;
    memcpy(&b, &hi, sizeof b);
    int e = static_cast<int>((b >> 23) & 0xFFu);
    if (e == 0) e = 1;
    const uint64_t d = static_cast<uint64_t>(166 - e + 1023) << 52;
    double r;
    memcpy(&r, &d, sizeof r);
    return r;
}
__host__ __device__ inline double v_join(float hi, int16_t lo) {
    return static_cast<double>(hi) + static_cast<double>(lo) * vlo_unit(hi);
}
__host__ __device__ inline void v_split(double v, float& hi, int16_t& lo) {
    hi = static_cast<float>(v);
    double q = rint((v - static_cast<double>(hi)) * vlo_inv_unit(hi));
    if (!(q >= -32768.0 && q <= 32767.0)) q = q > 0.0 ? 32767.0 : -32768.0;  // |q| <= 2^15; NaN -> bound
    lo = static_cast<int16_t>(q);
}
// the residual rows of a mixed velocity array
__host__ __device__ inline int16_t* v_lo_rows(void* v, int64_t nn_pad) {
    return reinterpret_cast<int16_t*>(static_cast<float*>(v) + 3 * nn_pad);
}

// Vector access to W consecutive entries of a padded SoA row (rows start
// 256-byte aligned, the row stride is a multiple of 32 entries and the first
// index a multiple of W): 16-byte chunks, or one 8-byte chunk when the W
// entries take 8 bytes.
template <int W, typename T>
__device__ __forceinline__ void ld_row(const T* p, T (&o)[W]) {
    constexpr int kBytes = W * static_cast<int>(sizeof(T));
    static_assert(kBytes % 16 == 0 || kBytes == 8 || kBytes == 4, "16-byte chunks or one 8- or 4-byte chunk");
    if constexpr (kBytes == 4) {
        const uint32_t q = *reinterpret_cast<const uint32_t*>(p);
        memcpy(o, &q, 4);
    } else if constexpr (kBytes == 8) {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        memcpy(o, &q, 8);
    } else {
#pragma unroll
        for (int i = 0; i < kBytes / 16; ++i) {
            const uint4 q = reinterpret_cast<const uint4*>(p)[i];
            memcpy(reinterpret_cast<char*>(o) + 16 * i, &q, 16);
        }
    }
}
template <int W, typename T>
__device__ __forceinline__ void st_row(T* p, const T (&v)[W]) {
    constexpr int kBytes = W * static_cast<int>(sizeof(T));
    static_assert(kBytes % 16 == 0 || kBytes == 8 || kBytes == 4, "16-byte chunks or one 8- or 4-byte chunk");
    if constexpr (kBytes == 4) {
        uint32_t q;
        memcpy(&q, v, 4);
        *reinterpret_cast<uint32_t*>(p) = q;
    } else if constexpr (kBytes == 8) {
        uint2 q;
        memcpy(&q, v, 8);
        *reinterpret_cast<uint2*>(p) = q;
    } else {
#pragma unroll
        for (int i = 0; i < kBytes / 16; ++i) {
            uint4 q;
            memcpy(&q, reinterpret_cast<const char*>(v) + 16 * i, 16);
            reinterpret_cast<uint4*>(p)[i] = q;
        }
    }
}
// W (2 or 4) consecutive bytes as one word, byte j of node j in bits 8j..8j+7.
template <int W>
__device__ __forceinline__ uint32_t ld_bytes(const uint8_t* p) {
    static_assert(W == 2 || W == 4, "2 or 4 bytes");
    if (W == 4) return *reinterpret_cast<const uint32_t*>(p);
    return *reinterpret_cast<const uint16_t*>(p);
}

// A NodeView of a batch table through the non-coherent (L1-cached) path:
// the table does not change while a pass runs.
__device__ __forceinline__ NodeView ld_view(const NodeView* p) {
    constexpr int kW = sizeof(NodeView) / sizeof(uint4);
    uint4 w[kW];
#pragma unroll
    for (int i = 0; i < kW; ++i) w[i] = __ldg(reinterpret_cast<const uint4*>(p) + i);
    NodeView v;
    memcpy(&v, w, sizeof(v));
    return v;
}
__device__ __forceinline__ NodeParam ld_param(const NodeParam* p) {
    uint4 w[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) w[i] = __ldg(reinterpret_cast<const uint4*>(p) + i);
    NodeParam v;
    memcpy(&v, w, sizeof(v));
    return v;
}
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Read-only input loads: through the non-coherent path from global memory,
// plain loads from a shared-memory stage.
template <bool SMEM, typename T>
__device__ __forceinline__ T ldin(const T* p) {
    if constexpr (SMEM) return *p;
    else return __ldg(p);
}

// The node pass's scalars of one batch slot: this cycle's stable dt
// (update_minVertex_perMaterial_and_dt, exDyna3D.cpp:673-679, as the
// single-instance node pass computes it), the previous dt and the gravity
// amplitude; also the control-block updates that pass makes.  Run by the
// last block of the batched element pass, after every block's minima: the
// edge minimum is read through L2.
__device__ inline void node_params_slot(const BatchTables& T, int slot) {
    const InstanceDesc& d = T.desc[slot];
    NodeParam p{0.0, 0.0, 1.0, 0, 0};
    Ctl* ctl = d.ctl;
    if (d.active && !ctl->done) {
        double dt_i;
        const int dt_final = ctl->dt_final;
        if (dt_final) {
            dt_i = ctl->dt_i;
        } else {
            double dd = __longlong_as_double(static_cast<long long>(__ldcg(&ctl->len_min))) / ctl->wos;
            const double tmp = ctl->dts_cur;
            dd = dd < tmp ? dd : tmp;
            dt_i = dd * ctl->factor;
        }
        if (!(dt_i > 0.0) || !isfinite(dt_i)) atomicOr(&ctl->status, ST_BAD_DT);
        if (!dt_final) ctl->dt_i = dt_i;
        ctl->cycles_done += 1;
        ctl->energy_pending = 1;
        p.dt_i = dt_i;
        p.dt_i_1 = ctl->dt_i_1;
        p.amp = (d.M.gravity_on && d.M.amp_n > 0) ? gravity_amplitude(d.M.amp, d.M.amp_n, ctl->time, dt_i) : 1.0;
        p.live = 1;
    }
    T.nparam[slot] = p;
}

// Called by every block of a batched element pass after its last tile: the
// last block to finish fills the node pass's scalars of all slots.
__device__ inline void element_pass_done(const BatchTables& T) {
    __shared__ int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(T.elem_done, 1) == static_cast<int>(gridDim.x) - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int slot = threadIdx.x; slot < T.counts[2]; slot += blockDim.x) node_params_slot(T, slot);
    if (threadIdx.x == 0) *T.elem_done = 0;
}

// Positive doubles order like their bit patterns; min-reductions over
// element dt / edge lengths use integer atomicMin on the bits, which is
// exact and independent of scheduling.
__device__ __forceinline__ unsigned long long ord_bits(double d) {
    return static_cast<unsigned long long>(__double_as_longlong(d));
}
__device__ __forceinline__ double bits_ord(unsigned long long b) {
    return __longlong_as_double(static_cast<long long>(b));
}
constexpr unsigned long long kInfBits = 0x7FF0000000000000ull;

}  // namespace ensc
