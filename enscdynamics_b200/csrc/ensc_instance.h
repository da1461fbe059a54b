// Host-side preparation and device layout of one solver instance, shared by
// the single-instance handle (ensc_capi.cu) and the batch (ensc_batch.cu).
// Internal; not part of the ABI.
#pragma once

#include "ensc_gpu.h"
#include "ensc_device.cuh"

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace ensc {

// Everything exDyna3D::init() derives from the deck before stepping
// (Explicit3D/source/exDyna3D.cpp:105-142) that the device needs, in host
// memory, plus the byte layout of the instance's device block.
struct InstanceHost {
    int64_t nn = 0, ne = 0, nn_pad = 0, ne_pad = 0;
    bool mixed = false, plastic = false, clash = false;
    std::vector<uint32_t> conn_soa;   // [8][ne_pad]
    std::vector<double> bt;           // [ne][24] row-major B0^T
    std::vector<double> vol0, cb, cb2;  // [ne] V0, cbrt(V0), cbrt(V0^2)
    std::vector<double> im;           // [nn_pad] inverse lumped mass per node
    std::vector<uint32_t> ell;        // [8][nn_pad] element in slot k, or ENSC_NONE
    std::vector<uint8_t> slot_mask;   // [nn_pad] occupied slots (clash-free meshes)
    std::vector<int64_t> csr_ptr;     // clash meshes: (slot, element)-sorted lists
    std::vector<uint32_t> csr_ent;
    const double* x0 = nullptr;       // caller arrays, read by instance_prepare only
    const double* v0 = nullptr;
    // the rows the upload copies as they are, formed by instance_prepare (so
    // that a prepared instance's host work is done before its device part):
    // mixed: A float pairs [18][ne_pad], cbrt(V0) as float [ne], v float
    // rows [3][nn_pad] and their 16-bit residual rows [3][nn_pad]; FP64:
    // B0^T [24][ne_pad], v [3][nn_pad]; both: x0 [3][nn_pad] (v rows empty
    // when the mesh has no initial velocities)
    std::vector<float> a_rows, cb_f, v_rows_f;
    std::vector<int16_t> v_lo_rows;
    std::vector<double> bt_rows, x_rows, v_rows_d;
    // patch assembly (ElemArrays::patch): the stored order of the elements
    // and the patch tables; all element arrays above are in stored order
    bool patch = false;
    std::vector<int32_t> iperm;       // [ne] element of the caller's numbering -> stored position
    std::vector<uint32_t> pf_off;     // [n_patches + 1]
    std::vector<uint32_t> pinc_off;   // [n_pnodes + 1]
    std::vector<uint16_t> pinc;       // [8 ne]
    std::vector<uint32_t> nptr;       // [nn + 1]
    std::vector<uint32_t> nent;       // [n_pnodes]
    int64_t n_patches = 0, n_pnodes = 0;
    // device layout: byte offsets of the pieces in one 256-byte-aligned block
    enum Piece {
        CONN, BT, VOL0, CB, CB2, SIG, QIA, EPS, FE, X, U, V, IM, BC, BCV, ELL, RF, CPTR, CENT, MASK,
        IPERM, PFOFF, PINCOFF, PINC, PF, NPTR, NENT, NPIECE
    };
    size_t off[NPIECE] = {};
    size_t size[NPIECE] = {};
    size_t bytes = 0;
};

// Validates the mesh and fills `h` (element constants computed as
// compute_invMassMatrix does unless the caller supplies them).
int instance_prepare(const ensc_mesh_desc* mesh, const ensc_material* mat, bool mixed, int assembly,
                     InstanceHost& h, std::string& err);

// Stored order of the patch assembly: elements sorted by the Morton key of
// their centroid's cell on a grid of the smallest element extent per axis,
// so that runs of kPatchElems stored elements are compact clusters.  Returns
// perm[stored position] = element of the caller's numbering.
std::vector<int32_t> patch_order(int64_t ne, const uint32_t* conn, const double* x0);

// Builds the patch tables of h (pf_off, pinc_off, pinc, nptr, nent) for the
// stored connectivity conn [ne][8].
void build_patches(int64_t nn, int64_t ne, const uint32_t* conn, InstanceHost& h);

// Copies the instance into `block` (h.bytes bytes, 256-byte aligned) on
// stream `st`, waits for the copies, and fills the array descriptors (PA
// all null under the slot assembly).
int instance_upload(const InstanceHost& h, void* block, cudaStream_t st, ElemArrays& E, NodeArrays& N,
                    PatchArrays& PA, std::string& err);

// Material_elastic::update (Material_elastic.cpp:9-14) plus the controls.
void material_from(const ensc_material* mat, const ensc_params* p, Material& M);

// Initial control block for time 0.
Ctl initial_ctl(const ensc_params* p, const Material& M);

}  // namespace ensc
