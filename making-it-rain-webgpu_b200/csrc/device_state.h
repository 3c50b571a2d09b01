// device_state.h -- the device tables of one engine, passed by value to every
// kernel, and the host-side launchers each kernel file provides.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace mdb {

// r0sq_hi + r0sq_lo is r0^2 to about 48 bits (an unevaluated f32 pair).
struct BondDev { int a, b, sys; float r0, k, r0sq_hi, r0sq_lo; };
struct AngleDev { int a, b, c, sys; float theta0, k; };
struct TorsionDev { int a, b, c, d, sys, periodicity; float phase, k; };
// qq values already carry ONE_4PI_EPS0 (kJ/mol nm).
struct ExceptionDev { int a, b, sys; float qq_particles, qq_own, sigma, eps4; };
struct RestraintDev { int p, sys; float k; long long x0, y0, z0; };

// One CTA of an FFT pass: system, first line (or x / y), kz start, count.
struct FftWork { int sys, a, b, n; };

struct Dev {
  int S;
  const SysDev* sys;
  RunDev run;
  int n_atoms, n_slots, n_blocks, n_cells, n_units, n_iblk;
  int cluster;        // atoms per cluster of the tile list: 8 or 32 (n_blocks counts clusters)
  int prune;          // rebuilds drop tiles with no pair inside cutoff + skin
  int inner;          // the pair kernel reads the inner list (see in_tiles)
  int any_triclinic;  // some system's box is triclinic: the pair kernel takes the general minimum image
  // nullptr, or per system 1 if the force kernels should compute it: an
  // evaluation of some of the systems (a barostat round's proposals) skips the others
  const unsigned char* active;

  // atoms, original order
  long long *px, *py, *pz;
  float *vx, *vy, *vz;
  float *rx, *ry, *rz;
  float* invm;
  int* atom_sys;
  int* rank;      // slot of an atom within its system's sorted order
  int* cell_of;   // global cell
  long long *refx, *refy, *refz;
  long long *bx, *by, *bz;         // positions before a Monte Carlo volume move
  const int* mol_off;              // molecule m's atoms: mol_atoms[mol_off[m] .. mol_off[m+1])
  const int* mol_atoms;            // global atom indices, molecule by molecule, system by system
  const float4* prm_atom;  // q*sqrt(ONE_4PI_EPS0), sigma/2, sqrt(24 eps), q

  // slots, sorted order
  int* order;     // global atom or -1
  // the order as the last integrator step saw it, kept only when the PME
  // spread goes by slot (spread_sorted): the spread reads this copy
  int* spread_atom;
  int spread_sorted;
  int* tmp_order;
  int4* pc;
  float4* prm;
  unsigned long long *fx, *fy, *fz;
  const int* slot_sys;

  // blocks
  float4 *bb_lo, *bb_hi;  // per cluster
  float4 *sb_lo, *sb_hi;  // per 32-slot super-cluster (the cluster boxes themselves when clusters are 32)
  int* fold;              // per slot: the lattice translation of the last rebuild's fold (3 x 10 bits)
  int2* raw_tiles;        // the fill pass's list, before pruning
  unsigned int* raw_masks;
  int4* raw_shift;
  unsigned char* tile_alive;  // per raw tile: some pair within cutoff + skin
  int* row_alive;         // per cluster: surviving tiles of its row
  int* alive_start;       // per cluster: their start after pruning
  int4* tile_shift;       // per tile: lattice shift of J in pair-coordinate units; w = 1: per-pair minimum image
  int* tile_cnt;
  int* tile_start;
  const int* block_sys;

  // cells
  int *cell_cnt, *cell_start, *cell_cur;
  const int* cell_sys;
  const int* cell_map;

  // tiles
  int2* tiles;
  unsigned int* masks;
  int* tile_count;   // per system
  int* tile_need;    // per system: tiles the last rebuild found (above tile_cap: it overflowed)
  int* tile_prefix;  // S+1
  int tile_cap_total; // sum of the systems' tile capacities
  int* halt;          // set when a list overflowed: the integrator stops advancing until the host rebuilds

  // inner list: the outer list's tiles that have a pair inside cutoff + inner
  // skin, in each system's region of the same capacity; the pair kernel's list
  // when `inner` is set.  Rebuilt from the outer list (copies of the tile, its
  // mask words and its shift) at every rebuild and whenever an atom has moved
  // half the inner skin since the last prune.
  int2* in_tiles;
  unsigned int* in_masks;
  int4* in_shift;
  int* in_count;      // per system
  int* in_prefix;     // S+1
  long long *prx, *pry, *prz;  // positions at the last prune, by atom
  float4 *cb_lo, *cb_hi;       // per cluster: bounding box at the last prune (pair coordinates, nm)
  int* prune_flag;    // set by the integrator: some atom moved inner skin/2
  int* prune_now;     // snapshot the list kernel acts on
  int* any_prune;
  long long* prune_count;  // per system: prunes between rebuilds
  int* inner_ticket;       // blocks of the inner-list kernel that have finished

  // flags and status
  int* rebuild_flag;  // set by the integrator: some atom moved skin/2
  int* rebuild_now;   // snapshot the rebuild kernels act on
  int* any_rebuild;
  int* err;           // per system ErrorBit
  long long* rebuild_count;
  int* global_ticket;
  unsigned int* list_barrier;  // count, generation: the cooperative list kernel's grid barrier

  // exclusions (every exception pair)
  const int2* excl;
  const int* excl_sys;
  int n_excl;

  // listed interactions
  const BondDev* bonds; int n_bonds;
  const AngleDev* angles; int n_angles;
  const TorsionDev* torsions; int n_torsions;
  const ExceptionDev* exceptions; int n_exceptions;
  const RestraintDev* restraints; int n_restraints;

  // PME
  unsigned long long* qgrid;
  float2* cgrid;
  float* phi;
  const float* moduli;
  const float2* twiddles;
  double* mesh_partial;  // one per x-pass work item
  double* mesh_virial;   // six per x-pass work item: xx yy zz xy xz yz
  const FftWork* fft_z; int n_fft_z;
  const FftWork* fft_y; int n_fft_y;
  const FftWork* fft_x; int n_fft_x;
  const FftWork* fft_p; int n_fft_p;  // whole x-planes (sys, x): the fused z+y passes, when they fit
  int fft_planes;                     // 1: the plane kernels replace the separate z and y passes
  float* influence;                   // per x-pass work item: its elements' influence function (k_influence)
  int influence_stride;               // floats per work item: kFftTile x the largest Kx

  // energies, int64 2^32 fixed, [S][kECount]
  unsigned long long* energy;

  // integrator
  const UnitDev* units;
  const int* iblk_sys;
  const int* iblk_unit0;
  const int* iblk_nunit;
  const int* iblk_atom0;  // first table entry of each integrate block in `iatom`
  const int* iblk_natom;
  const int* iatom;       // global atom index of every table entry, block by block
  double* mom_partial;  // 3 per integrate block
  float4* vcom;         // per system, for the next step's COM removal
  long long* step;      // per system
  int* done_count;      // per system
  int* shake_failures;
};

__device__ __forceinline__ bool sys_active(const Dev& d, int s) { return d.active == nullptr || d.active[s] != 0; }

// ---- chained launches (programmatic dependent launch) ----
// A kernel launched by `launch_chained` may begin before the kernel ahead of
// it in its stream has finished: its blocks become resident once every block
// of that kernel has called `release_successor` or exited, and they wait in
// `wait_for_predecessor` until it has finished and its writes are visible.
// Every kernel launched this way calls wait_for_predecessor first, before any
// global memory access; launched normally the wait returns at once.  The PME
// chain and the integrator release only by exiting: blocks released early sit
// on SMs the pair kernel beside them could use (octahedron step 0.152 against
// 0.143 ms with early releases).  Measured against plain launches: peptide
// step 0.0952 against 0.0975 ms, octahedron 0.1431 against 0.1451 ms.
__device__ __forceinline__ void wait_for_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void release_successor() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... P, typename... A>
void launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<A&&>(args)...);
}

constexpr int kFftTile = 8;  // kz columns per y- and x-pass CTA of the PME transform

// ---- launchers (one per kernel file) ----
int prepare_list_kernel(int device);                      // 0: no cooperative launch
bool launch_list(const Dev& d, cudaStream_t s);            // sort + wrap + tiles, one launch
void launch_rebuild_sort(const Dev& d, cudaStream_t s);     // phases 0-4
void launch_wrap(const Dev& d, cudaStream_t s);
void launch_rebuild_tiles(const Dev& d, cudaStream_t s);    // phases 5-9
void launch_inner_prune(const Dev& d, cudaStream_t s);      // the inner list, when one is due
void launch_nonbonded(const Dev& d, bool energy, cudaStream_t s);
void launch_listed(const Dev& d, bool energy, cudaStream_t s);
void launch_pme(const Dev& d, bool energy, cudaStream_t s);
bool spread_by_slot(int n_slots);  // whether an engine of n_slots slots spreads PME charges by slot
void launch_pme_spread(const Dev& d, cudaStream_t s);
void launch_pme_fft(const Dev& d, bool energy, cudaStream_t s);
void launch_pme_gather(const Dev& d, cudaStream_t s);
void launch_influence(const Dev& d, int sys, cudaStream_t s);  // after a box change; sys < 0: every system
void launch_integrate(const Dev& d, cudaStream_t s);
void launch_momentum(const Dev& d, cudaStream_t s);
void launch_scale_molecules(const Dev& d, int first_mol, int n_mol, double scale, cudaStream_t st);
void launch_restore_positions(const Dev& d, int atom_off, int n, cudaStream_t st);
void launch_after_box_change(const Dev& d, int s, int n_slots, int tile_cap, cudaStream_t st);
int molecular_offset_blocks(int n_mol);
void launch_molecular_offsets(const Dev& d, int first_mol, int n_mol, int slot_off, double* partials,
                              cudaStream_t st);

}  // namespace mdb
