// Batched SCF: many molecules of uneven size advanced together, one launch per SCF phase.
//
// Every molecule owns one device allocation holding its geometry tables, stored pair
// integrals, core Hamiltonian, densities and DIIS history (MolDesc points into it) and a
// control record (MolCtl) that the device updates: the DIIS ring bookkeeping, the A-DIIS /
// CDIIS weights, the stall guard and the convergence test of pm7-rs src/scf.rs:1189-1322,
// 1534-1916 run per molecule on the device, so an SCF iteration of the whole batch needs
// no host decision. A phase kernel takes the list of active molecules and the exclusive
// prefix of their work-item counts; a block maps its item to (molecule, local item) by
// binary search, so molecules of any size share one launch.
#pragma once

#include <cstdint>

#include "kernels.hpp"

namespace pm7 {

constexpr int kHist = 8;  // DIIS depth (scf.rs:1189-1322)

// One molecule as the batched kernels see it (device memory; fixed after admission).
struct MolDesc {
  FockGeometry g;            // atoms, AO layout, near pairs, w store, near mask
  int n_occ, dframe, cc_nx;  // cc_nx: column blocks of the core-core sweep (ceil(N/128))
  int want_matrices, smooth_dispersion;
  double *H, *w, *ecore, *jbuf, *pop;  // w: writable alias of g.w
  double *cc_terms;          // build only: pair core-core energies in pair order (aliases X)
  double *P, *Pn, *X;        // density, next density, scratch (nao^2 each; P/Pn swap on device)
  double *hist;              // kHist x {F, E = FP - PF, D} blocks of nao^2
  double *eps_out, *V_out;   // reported orbital energies (nao) and vectors (nao^2, optional)
  double *atom_out;          // per atom: population and the hybrid-dipole density elements
  double *part;              // per-item partial sums of the chunked reductions (kPart each)
  float *X32, *hi32, *lo32, *C32;  // mixed precision: fp32 SP2 iterate, its tf32 split, X^2 (ld32^2)
  float *P32, *w32;          // mixed precision: the density and the w store as float (FP32 Fock build)
  size_t w_len;              // doubles in the w store
  int ld32;
  double *corr_scratch;      // post-SCF corrections scratch
};

constexpr int kAtomOut = 16;  // doubles per atom in MolDesc::atom_out

// Per-molecule SCF control state (device memory, updated only by the control kernels).
struct MolCtl {
  // options (scf.rs:207-233)
  int max_scf, accel;  // accel: 0 none, 1 A-DIIS with CDIIS switch, 2 CDIIS only
  double e_tol, p_tol, adiis_switch, shift_floor;
  // progress
  int iter, done, converged, slot;
  int n_ord, ord[kHist];
  double gram[kHist * kHist], xdf[kHist * kHist];
  double e_elec, e_old, err2, dp, shift;
  int n_win;
  double win_step[10], win_e[10];
  // extrapolation of this iteration: sum_i coef[i] F_{csrc[i]}
  int ncoef, csrc[kHist];
  double coef[kHist];
  // inner products of this iteration (see k_b_dots)
  double ee[kHist + 1], df_row[kHist + 1], df_col[kHist];
  // SP2 purification of this iteration: state 0 running, 1 converged, 2 failed
  int sp2_state, sp2_steps, sp2_fallbacks, sp2_square, sp2_apply;
  int mixed, use32, fp32_iters;  // mixed precision: still in fp32 cycles, this cycle fp32, count
  int f32_slots;                 // ring slots whose Fock matrix came from the FP32 build (bit mask)
  double sp2_err[3], sp2_emin, sp2_emax;
  // results
  double core_core, e_final, corr[5];
  double e_fold[2];  // <P, H> and <P, F> of the final density, as the reference's folds
};

// Where this iteration's eigensolve of a molecule lives (bucket buffers, row k of V =
// eigenvector k, row stride ldv; `in` receives the extrapolated Fock, padded).
struct EigSlot {
  double *in, *eps;
  int ldv, pad_;
};

// Active molecules of one launch and the exclusive prefix of their work-item counts.
struct BatchList {
  const int *slot;    // molecule slot of list position m
  const int *prefix;  // prefix[m] = first item of position m; prefix[n] = total
  int n;
  int total;          // prefix[n], known to the host that built the list
};

// Largest m with prefix[m] <= item.
__device__ __forceinline__ int batch_find(const BatchList &L, int item) {
  int lo = 0, hi = L.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (L.prefix[mid] <= item) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ size_t mol_nn(const MolDesc &d) { return (size_t)d.g.nao * d.g.nao; }
__device__ __forceinline__ double *hist_F(const MolDesc &d, int s) { return d.hist + (size_t)s * 3 * mol_nn(d); }
__device__ __forceinline__ double *hist_E(const MolDesc &d, int s) { return hist_F(d, s) + mol_nn(d); }
__device__ __forceinline__ double *hist_D(const MolDesc &d, int s) { return hist_F(d, s) + 2 * mol_nn(d); }

// Whether this iteration's Fock build of a molecule runs in FP32: a mixed-precision molecule
// in its fp32 cycles whose DIIS error is above kFock32Switch eV (the guess and the first A-DIIS
// cycles). The SCF does not end while the DIIS history holds such a Fock matrix.
constexpr double kFock32Switch = 10.0;
__device__ __forceinline__ bool fock32_now(const MolDesc &d, const MolCtl &c) {
  return d.P32 != nullptr && c.mixed && (c.iter == 0 || c.err2 > kFock32Switch * kFock32Switch);
}

// Chunk `item` of a chunk list: list position, slot and element range [e0, e1).
struct ChunkRef {
  int m, slot, q;
  size_t e0, e1;
};
constexpr int kChunkElems = 32768;
__device__ __forceinline__ ChunkRef chunk_ref(const BatchList &L, const MolDesc *D, int item) {
  ChunkRef r;
  r.m = batch_find(L, item);
  r.slot = L.slot[r.m];
  r.q = item - L.prefix[r.m];
  const size_t nn = mol_nn(D[r.slot]);
  r.e0 = (size_t)r.q * kChunkElems;
  r.e1 = r.e0 + kChunkElems < nn ? r.e0 + kChunkElems : nn;
  return r;
}

// ---- batched phase launchers (kernels_*.cu) ----
// Work items per molecule, for building the prefix arrays on the host.
inline int items_pairs_all(int n_atoms) { return n_atoms * ((n_atoms + 127) / 128); }
inline int items_near_chunks(int n_near) { return (n_near + 127) / 128; }
inline int items_gemm_full(int nao) { const int t = (nao + 63) / 64; return t * t; }
inline int items_gemm_lower(int nao) { const int t = (nao + 63) / 64; return t * (t + 1) / 2; }
inline int items_rows8(int nao) { return (nao + 7) / 8; }
// Matrix-element chunks of the elementwise and reduction kernels: a large molecule is
// spread over many blocks; each chunk leaves kPart partial sums that a per-molecule pass
// adds in chunk order.
constexpr int kChunk = kChunkElems;
constexpr int kPart = 32;
__host__ __device__ inline int items_chunks(int nao) {
  return (int)(((size_t)nao * nao + kChunk - 1) / kChunk);
}
constexpr int kDPairsPerBlock = 2;
inline int items_near_d(int n_near) { return (n_near + kDPairsPerBlock - 1) / kDPairsPerBlock; }

void launch_b_pairs_all(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P);
void launch_b_pairs_all_d(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P);
void launch_b_near_integrals(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P);
void launch_b_near_integrals_d(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P);
// items: atoms
void launch_b_hcore_diag(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P);

// Fock of every listed molecule from its density P: into the history slot ctl.slot
// (final = 0) or into X (final = 1). Lists: per molecule (pop), rows of 8 (far), near
// chunks, atoms.
void launch_b_fock(cudaStream_t st, const BatchList &Lmol, const BatchList &Lrows, const BatchList &Lnear,
                   const BatchList &Latoms, const MolDesc *D, const MolCtl *C, const DeviceParams &P, int final_pass);

// op 0: X = F_slot P (full tiles); op 1: Pn = 2 V_occ^T V_occ (lower tiles, mirrored);
// op 2: Pn = X X for molecules whose SP2 purification is still running (lower tiles).
void launch_b_gemm(cudaStream_t st, const BatchList &L, const MolDesc *D, const MolCtl *C, const EigSlot *E, int op);

// Mixed precision (kernels_tf32.cu): items_tiles128 per molecule for the squaring; chunks
// for the conversions and updates; one block per molecule for the decisions.
inline int items_tiles128(int nao) { const int t = (nao + 127) / 128; return t * (t + 1) / 2; }
void launch_b_square_tf32x3(cudaStream_t st, const BatchList &L, const MolDesc *D, const MolCtl *C,
                            const void *maps, int *error);
void launch_b_to32(cudaStream_t st, const BatchList &L, const MolDesc *D);
void launch_b_sp2_decide32(cudaStream_t st, const BatchList &L, const MolDesc *D, MolCtl *C, unsigned char *flags);
void launch_b_sp2_apply32(cudaStream_t st, const BatchList &L, const MolDesc *D, const MolCtl *C);

// Post-SCF corrections of the listed molecules into C[slot].corr (dispersion variant per
// molecule from MolDesc::smooth_dispersion). Lmol: one item per molecule; Lpairs:
// items_pairs_all(n_atoms) per molecule; max_atoms over the list.
void launch_b_corrections(cudaStream_t st, const BatchList &Lmol, const BatchList &Lpairs, const MolDesc *D, MolCtl *C,
                          int method, int max_atoms);

}  // namespace pm7
