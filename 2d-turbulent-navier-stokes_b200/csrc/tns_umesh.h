// tns_umesh.h -- general quadrilateral meshes: the device view of a mesh that is not one
// structured i x j block, and the runtime entry points of tns_unstructured.cu.
//
// The reference works on any quad connectivity (geometry.f90:31-52 reads NOD(:,1:4) and
// NC1..NC4 as given; every stencil gathers through NCk(I)).  Such a mesh is laid out
// with its cells in the order of their centroids along a Hilbert curve, so that the
// neighbours a cell gathers sit close in memory and each run of 256 cells is a compact
// chunk with a short halo; ghosts are slots NE..NE+NGHOSTS-1 in bc.in order, nodes are
// renumbered in the order the cells first reach them.  Kernels gather through index
// arrays; the RK stages stage each chunk and its halo in shared memory.
#pragma once

#include <cuda_runtime.h>

#include "../../include/tnsgpu.h"
#include "tns_device.cuh"

struct tns_handle;

namespace tns {

// Static per-cell geometry [UCG_N][ne] (geometry.f90:55-149 with the gradient
// coefficients of source_terms.f90:24-60, as in source_terms()).
enum UCellGeo {
    UCG_SX1, UCG_SX2, UCG_SX3, UCG_SX4, UCG_SY1, UCG_SY2, UCG_SY3, UCG_SY4,
    UCG_GA, UCG_GB, UCG_GC, UCG_GD, UCG_VOL, UCG_RVOL, UCG_YCC, UCG_RYCC, UCG_N
};
// Static geometry of face k (0..3) of each cell for the viscous flux (viscous.f90:130-217,
// A = the cell, C = NC_k, B = node N_k, D = node N_k+1): [UFG_N][4][ne], the
// diamond-gradient coefficients and 1/YAVG (0 where YAVG is below the axis threshold).
enum UFaceGeo { UFG_GA, UFG_GB, UFG_GC, UFG_GD, UFG_RYAVG, UFG_N };
// Per-slot (cells, then ghosts) primitive and flux field set of one stage [UW_N][ne+ng].
enum USlot {
    UW_F1, UW_F2, UW_F3, UW_F4, UW_F5, UW_G1, UW_G2, UW_G3, UW_G4, UW_G5,
    UW_U, UW_V, UW_T, UW_P, UW_RHO, UW_RI, UW_QM, UW_N
};

struct UMesh {
    int ne, ng, nnode, nport;
    const int* nc;        // [4][ne] neighbour slot: a cell 0..ne-1 or a ghost ne+line
    const int* nod;       // [4][ne] 0-based node ids
    const double* cg;     // [UCG_N][ne]
    const double* fg;     // [UFG_N][4][ne]
    const double* cfldl;  // [ne] CFL*DL
    const int* gpar;      // [ng] parent cell
    const int* gopp;      // [ng] the parent's neighbour across the face opposite the ghost
    const int* gtype;     // [ng] BC type
    const int* gside;     // [ng] NSIDE
    const double* gsx;    // [ng] the parent's face vector on the ghost's side
    const double* gsy;
    const double* gyc;    // [ng] mirrored ghost centroid y (geometry.f90:114-142)
    const double* ginj;   // [ng] type-6 burn-rate multiplier
    double* gport;        // [ng] type-6 port mass flux of the current stage input
    const int* nptr;      // [nnode+1] contributions of each node (cells by id, then ghosts)
    const int* nslot;     // contributing slot
    const int* nreset;    // 0, or the BC type (4, 5) whose reset follows the contribution
    const int* pghost;    // [nport] ghost line of each type-6 ghost
    const int* pptr;      // [nport+1] the cells of its port line, from the parent across
    const int* pcell;
    const double* pdely;  // DELY of each of those cells for the ghost's side
    // viscous faces: each face evaluated once, in the orientation of its owner cell (the
    // lower id of two cells; the cell of a ghost face); fcell[e] = 4 * owner + face, and
    // per cell face fref[k][ne] = e (the cell owns it) or ~e (its neighbour does: the cell
    // adds -F_e)
    int nface;
    const int* fcell;
    const int* fref;
    // stage chunks: chunk b holds cells UT b .. UT b + UT - 1 and the halo slots
    // cslot[cptr[b] .. cptr[b+1]) (cells of other chunks and ghosts its cells touch);
    // lnb[k][ne] is the local slot of each cell's face-k neighbour (below UT: a cell of
    // the chunk, UT + h: halo slot h); hmax the largest halo
    int nchunk, hmax;
    const int* cptr;
    const int* cslot;
    const int* lnb;
};
constexpr int UT = 256;  // threads per block of the general-mesh kernels, cells per stage chunk

struct StageArgsU {
    const double* qold;  // [5][ne] state at the start of the iteration
    double* qout;        // [5][ne] stage output (may alias qold: own-cell reads only)
    const double* d;     // [5][ne]
    const double* vis;   // [4][ne]
    const double* dt;    // [ne] (LOCAL=1)
    const double* dtmin; // (LOCAL=0)
    double alpha;
    unsigned long long* cdiff;
    unsigned int* status;
};

void launch_u_prim(const Params& P, const UMesh& M, const double* q, double* W, cudaStream_t s);
// the same for the mixed path's stage input COLD + dQ (dq null: COLD)
void launch_u_prim_mx(const Params& P, const UMesh& M, const double* cold, const float* dq, double* W,
                      cudaStream_t s);
void launch_u_gport_mx(const Params& P, const UMesh& M, const double* cold, const float* dq, cudaStream_t s);
// mixed path: D, DT (dissipation) and VIS (viscous) stored in FP32
void launch_u_dissipation(const Params& P, const UMesh& M, const double* q, double* aux, float* d, float* dt,
                          const double* dtmin, cudaStream_t s);
void launch_u_viscous(const Params& P, const UMesh& M, const double* W, double* na, double* vf, float* vis,
                      cudaStream_t s);
void launch_u_gport(const Params& P, const UMesh& M, const double* q, cudaStream_t s);
void launch_u_dissipation(const Params& P, const UMesh& M, const double* q, double* aux, double* d,
                          double* dt, const double* dtmin, cudaStream_t s);
void launch_u_viscous(const Params& P, const UMesh& M, const double* W, double* na, double* vf, double* vis,
                      cudaStream_t s);
// one RK stage on state q, chunk by chunk; configure_u_chunk once per mesh
void launch_u_stage_chunk(const Params& P, const UMesh& M, const StageArgsU& A, const double* q, cudaStream_t s);
cudaError_t configure_u_chunk(const UMesh& M);
// the mixed FP32/FP64 stage (tns_unstructured_mx.cu): A.cold + A.dqin in, A.dqout or
// (stage 4) A.qout out; configure_u_chunk_mx once per mesh
struct StageArgsMx;
void launch_u_stage_chunk_mx(const Params& P, const UMesh& M, const StageArgsMx& A, cudaStream_t s);
cudaError_t configure_u_chunk_mx(const UMesh& M);
size_t u_chunk_mx_smem_bytes(const UMesh& M);
size_t u_chunk_smem_bytes(const UMesh& M);
void launch_u_post_average(const UMesh& M, const double* W, double* out, cudaStream_t s);
void launch_u_prim_out(const UMesh& M, const double* W, double* out, cudaStream_t s);
void launch_u_boundary_sums(const Params& P, const UMesh& M, const double* W, int type, int side,
                            int mode, double* out, cudaStream_t s);
void launch_u_face_states(const Params& P, const UMesh& M, const double* W, double* out, cudaStream_t s);

}  // namespace tns

namespace tns_rt {
// Host layout of a general mesh (after build_mesh found no structured block): validates
// the arrays as build_mesh does, renumbers the cells, computes the geometry.
int umesh_build(tns_handle* h, const tns_mesh* m);
int umesh_upload(tns_handle* h);
void enqueue_iteration_u(tns_handle* h, bool monitor);
// the mixed-precision iteration from state buffer A to Aout (FP32 increments between
// the stages, as the structured mixed path)
void enqueue_iteration_u_mx(tns_handle* h, bool monitor, double* A, double* Aout);
// U, V, T, P of cells and ghosts of the last stage's input into h->primout ([4][ne+ng],
// slot order)
int umesh_primitives(tns_handle* h);
int umesh_node_averages(tns_handle* h, double* dev_out);  // [4][nnode]: P, U, V, T
int umesh_boundary_sums(tns_handle* h, int type, int side, int mode, double* dev_out);
int umesh_face_states(tns_handle* h, double* dev_out);  // [5][ng], bc.in order
int umesh_set_injection(tns_handle* h, const double* scale);
void umesh_release(tns_handle* h);
}  // namespace tns_rt
