// Internal launcher declarations shared by the kernel translation units and
// the C-ABI implementation (ensc_capi.cu).  Not installed; not part of the ABI.
#pragma once

#include "ensc_device.cuh"

#include <string>

namespace ensc {

constexpr int kElemThreads = 128;

// Minimum resident blocks per SM requested from the compiler for the element
// passes (register budget = 65536 / (128 * minb)); tuned on B200.
#ifndef ENSC_ELEM_MINB_FP64
#define ENSC_ELEM_MINB_FP64 3
#endif
#ifndef ENSC_ELEM_MINB_MIXED
#define ENSC_ELEM_MINB_MIXED 6
#endif
// Unroll factor of the element passes' loops over the 8 nodes: more in-flight
// gathers per thread against more live registers.
#ifndef ENSC_NODE_UNROLL_FP64
#define ENSC_NODE_UNROLL_FP64 8
#endif
#ifndef ENSC_NODE_UNROLL_MIXED
#define ENSC_NODE_UNROLL_MIXED 4
#endif
constexpr int kNodeUnrollFp64 = ENSC_NODE_UNROLL_FP64;
constexpr int kNodeUnrollMixed = ENSC_NODE_UNROLL_MIXED;
// Mixed element pass with its streamed inputs staged in shared memory by
// bulk copies (k_element_mixed_staged) instead of per-thread loads.
#ifndef ENSC_STAGED_MIXED
#define ENSC_STAGED_MIXED 1
#endif
// elements per stage (= threads per block) and resident blocks per SM of
// the staged mixed pass; tuned on B200
#ifndef ENSC_STAGE_TILE_MIXED
#define ENSC_STAGE_TILE_MIXED 64
#endif
#ifndef ENSC_STAGE_MINB_MIXED
#define ENSC_STAGE_MINB_MIXED 8
#endif
#ifndef ENSC_BATCH_MINB_MIXED
#define ENSC_BATCH_MINB_MIXED 8
#endif
// 1: the staged mixed element passes read A and the connectivity from the
// stage again for the force step instead of keeping them in registers
#ifndef ENSC_MIXED_REREAD
#define ENSC_MIXED_REREAD 1
#endif
// The single-instance staged mixed element pass prefetches an element's node
// rows into L1 before its coordinate phase: bit 0 the velocities, bit 1 the
// coordinate components 1 and 2
#ifndef ENSC_MIXED_PREFETCH
#define ENSC_MIXED_PREFETCH 3
#endif
// The same for the batched mixed element pass, off: with the instance's
// arrays in registers the prefetch addresses spill (measured on B200: the
// velocity rows there spill 216 B per thread and cost 6%; with the
// addresses formed inside the prefetch instruction the spill is 36 B and the
// cost 4-6% on the block and on a 64-instance sweep)
#ifndef ENSC_BATCH_MIXED_PREFETCH
#define ENSC_BATCH_MIXED_PREFETCH 0
#endif
// how the batched mixed element pass reads the staged instance descriptor:
// 1 all fields copied to registers per tile, 2 arrays copied and material
// constants read at use, 0 everything read at use
#ifndef ENSC_BATCH_DESC_MODE
#define ENSC_BATCH_DESC_MODE 2
#endif
// 1: the grouped node passes sum all 8 force slots (empty ones hold zeros)
// instead of reading the slot mask first (measured on B200, mixed: reading
// the mask made the node pass 22% slower on the block and the batched
// 64-instance sweep of plates and cantilevers, whose many boundary nodes have
// empty slots, 5% slower)
#ifndef ENSC_NODE_ALL_SLOTS
#define ENSC_NODE_ALL_SLOTS 1
#endif
// 1: the mixed node passes load the nodes' own rows (v, its residual, x,
// the inverse mass, the BC code) before the force slots, so that all the
// group's loads are in flight together (measured on B200: node pass 4%
// faster, bit-identical)
#ifndef ENSC_NODE_LOAD_FIRST
#define ENSC_NODE_LOAD_FIRST 1
#endif
#ifndef ENSC_NODE_BATCH_MINB_MIXED
#define ENSC_NODE_BATCH_MINB_MIXED 2
#endif
// FP64 element pass staged the same way: 0 off, 1 staging all streamed
// inputs except B0^T (read from global memory), 2 staging B0^T too.
#ifndef ENSC_STAGED_FP64
#define ENSC_STAGED_FP64 2
#endif
// 1: the single-instance FP64 element pass runs one bulk-copy pipeline per
// warp (k_element_fp64_warp: 32-element tiles, two stages per warp, no
// block-wide barrier per tile) instead of one per block (measured on B200
// on the block workload: 0.6% faster; the same structure for the mixed
// passes was 1-3% slower than their per-block pipelines)
#ifndef ENSC_WARP_PIPE_FP64
#define ENSC_WARP_PIPE_FP64 1
#endif
#ifndef ENSC_F64_PIPE_WARPS
#define ENSC_F64_PIPE_WARPS 4
#endif
// 1: the warp-pipelined FP64 pass stages B0^T too; 0: reads it through L1
#ifndef ENSC_F64_WARP_BT
#define ENSC_F64_WARP_BT 1
#endif
// The FP64 warp-pipelined element pass prefetches an element's node rows
// into L1 once its connectivity is staged: bit 0 the velocities, bit 1 the
// displacements
#ifndef ENSC_F64_PREFETCH
#define ENSC_F64_PREFETCH 3
#endif
// elements per tile of the batched FP64 element pass, one block of as many
// threads per tile (32 would make every block one warp with its own
// two-stage pipeline, as in the single-instance pass: 2% slower on the
// 256-instance sweep, 0.6% faster on the block)
#ifndef ENSC_F64_BATCH_TILE
#define ENSC_F64_BATCH_TILE 128
#endif
#ifndef ENSC_F64_PIPE_MINB
#define ENSC_F64_PIPE_MINB 2
#endif
// elements per stage (= threads per block) of the staged FP64 passes
#ifndef ENSC_STAGE_TILE_FP64
#define ENSC_STAGE_TILE_FP64 128
#endif
constexpr int kNodeThreads = 256;
constexpr int kCtlThreads = 256;

// FP64 (ensc_fp64.cu, built with -fmad=false)
void launch_element_fp64(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                         int grid, bool init, cudaStream_t st);
void launch_node_fp64(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                      int grid, cudaStream_t st);
int occupancy_element_fp64(bool plastic);
// nodes per thread of the node pass on the padded slot-major layout
#ifndef ENSC_NODE_GROUP_MIXED
#define ENSC_NODE_GROUP_MIXED 4
#endif
// resident blocks per SM requested for the node passes (register budget
// 65536 / (256 * minb)); tuned on B200
#ifndef ENSC_NODE_MINB_MIXED
#define ENSC_NODE_MINB_MIXED 2
#endif
#ifndef ENSC_NODE_MINB_FP64
#define ENSC_NODE_MINB_FP64 4
#endif
constexpr int kNodeGroupFp64 = 2;
constexpr int kNodeGroupMixed = ENSC_NODE_GROUP_MIXED;
// nodes per thread of the batched mixed node pass (with the nodes' rows
// loaded first, 4 spill there; 2 were 1% faster on the block as a batch and
// on a 64-instance sweep than 4 without loading first)
#ifndef ENSC_NODE_GROUP_BATCH_MIXED
#define ENSC_NODE_GROUP_BATCH_MIXED 2
#endif
constexpr int kNodeGroupBatchMixed = ENSC_NODE_GROUP_BATCH_MIXED;
int node_group_width(bool mixed_precision);
int occupancy_node_fp64();

// mixed precision (ensc_mixed.cu)
void launch_element_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                          int grid, bool init, cudaStream_t st, const PatchArrays& PA = PatchArrays{});
void launch_node_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                       int grid, cudaStream_t st, const PatchArrays& PA = PatchArrays{});
int occupancy_element_mixed(bool plastic);
int occupancy_node_mixed();

// the last cycle's acceleration (compute_a), interleaved xyz per node, from
// the element forces the last force pass left in E.fe
void launch_acceleration_fp64(const ElemArrays& E, const NodeArrays& N, const Material& M, const Ctl* ctl,
                              double* a_aos, cudaStream_t st);
void launch_acceleration_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M, const Ctl* ctl,
                               double* a_aos, cudaStream_t st, const PatchArrays& PA = PatchArrays{});

// batched instances (one launch per phase for all instances of a batch)
void launch_element_batch_fp64(const BatchTables& T, int grid, cudaStream_t st);
// threads per block of the batched node passes: kNodeThreads or half of it
void launch_node_batch_fp64(const BatchTables& T, int grid, int threads, cudaStream_t st);
int occupancy_element_batch_fp64();
int occupancy_node_batch_fp64(int threads);
void launch_element_batch_mixed(const BatchTables& T, int grid, int ept, bool patch, cudaStream_t st);
void launch_node_batch_mixed(const BatchTables& T, int grid, int threads, bool patch, cudaStream_t st);
int occupancy_element_batch_mixed(int ept);
int occupancy_node_batch_mixed(int threads);
// elements and nodes per batch tile (element tiles are the staged passes'
// tiles; node tiles are one warp of node groups)
int batch_element_tile(bool mixed_precision);
int batch_element_tile_fp64();
int batch_node_tile(bool mixed_precision);
void launch_between_batch(const BatchTables& T, int slots, int mode, cudaStream_t st);
void launch_edge_prepass_batch(const BatchTables& T, int grid, cudaStream_t st);
// per-instance node-pass scalars (and the control-block updates of the node
// pass); runs between the element and node passes

// control (ensc_control.cu, built with -fmad=false)
// mode 0: fold energy partials + begin next cycle; 1: fold only; 2: fold as initial KE
void launch_between(Ctl* ctl, const Partials& P, int mode, cudaStream_t st);
void launch_edge_prepass(const ElemArrays& E, const NodeArrays& N, Ctl* ctl, int grid, cudaStream_t st);
// pause: the instance stops after the cycle in which its time reaches pause
// (dt is not clamped to it)
void launch_arm(Ctl* ctl, double step_end, long long max_cycles, cudaStream_t st, double pause = HUGE_VAL);
void launch_apply_bc_v(const NodeArrays& N, bool fp32_v, cudaStream_t st);
void launch_reset_init(Ctl* ctl, cudaStream_t st);
void launch_kinetic0(const NodeArrays& N, const Partials& P, Ctl* ctl, bool fp32_v, int grid, cudaStream_t st);
// layout conversion between caller AoS arrays and device SoA arrays
// `at` (may be null): entry e of the interleaved array is SoA row position
// at[e] -- an element's stored position under the patch order
void launch_soa_to_aos(const void* soa, int64_t n, int64_t pad, int comps, bool src_fp32, double* aos,
                       cudaStream_t st, const int32_t* at = nullptr);
void launch_aos_to_soa(const double* aos, int64_t n, int64_t pad, int comps, void* soa, bool dst_fp32,
                       cudaStream_t st, const int32_t* at = nullptr);
// displacements of a mixed instance (u rows holding xr = x - u) to
// interleaved xyz doubles; and a <- x - a over three node rows
void launch_disp_to_aos(const double* x, const double* xr, int64_t n, int64_t pad, double* aos, cudaStream_t st);
void launch_reflect_rows(const double* x, double* a, int64_t n, int64_t pad, cudaStream_t st);
// velocities (FP64 rows, or the mixed stepper's float rows and residual rows)
// to and from interleaved xyz doubles
void launch_v_to_aos(const NodeArrays& N, bool fp32_v, double* aos, cudaStream_t st);
void launch_aos_to_v(const double* aos, const NodeArrays& N, bool fp32_v, cudaStream_t st);

// thread-local message returned by ensc_last_error(NULL) (ensc_capi.cu)
void set_thread_error(const std::string& msg);

}  // namespace ensc
