// common.cuh -- device data layout and arithmetic shared by every kernel.
//
// Layout in HBM (all systems of a batch concatenated; every table carries
// per-system offsets in `SysDev`):
//   per atom, original order   positions int64 x/y/z (2^32 fixed point),
//                              velocities f32 x/y/z, drift residual f32 x/y/z,
//                              1/m f32, owning system, slot (rank) in the sorted
//                              order, reference positions at the last list build.
//   per slot, sorted order     atom index (-1 = padding), pair coordinates int4
//                              (int32 at 2^pc_shift per nm, folded into the
//                              cell), pair parameters float4, forces int64 x/y/z.
//   per 32-slot block          bounding box, tile-row count and start.
//   per tile (block pair)      (I, J) and 32 interaction-mask words.
//   PME                        int64 charge grid, f32 complex half spectrum,
//                              f32 potential grid, per-axis B-spline moduli.
// Everything is structure-of-arrays so that a warp reads 32 consecutive words.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mdb {

constexpr double kOne4PiEps0 = 138.93545764498457;  // src/engine/units.ts:18
constexpr double kBoltzmann = 0.008314462618153242;  // units.ts:15
constexpr int kTile = 32;
constexpr int kPmeOrder = 5;
constexpr int kMaxClusterAtoms = 8;
constexpr int kMaxClusterConstraints = 8;
constexpr int kMaxShakeIterations = 150;  // src/reference/constraints.ts:34
constexpr int kMaxRadices = 12;

// Per-system energy accumulators, int64 at the 2^32 fixed-point scale.
enum EnergySlot : int {
  kEBond = 0,
  kEAngle,
  kETorsion,
  kERestraint,
  kECoulomb,
  kELj,
  kEExclusion,
  kEException,
  kEVirial0,  // 9 virial components follow
  kEPairs = kEVirial0 + 9,  // in-cutoff pair count (an integer, not fixed point)
  kECount
};

// Device status bits, OR-ed into `err` and turned into C-ABI codes by the host.
enum ErrorBit : int {
  kErrTileCapacity = 1,
  kErrRange = 2,
  kErrShake = 4,
  kErrTimeout = 8,
  kErrCellCapacity = 16
};

// kUnitStar: a SHAKE cluster whose constraints all join atom 0 to atoms
// 1..nc (X-H_n, nc <= 3), solved with compile-time sizes.
enum UnitKind : int { kUnitFree = 0, kUnitSettle = 1, kUnitShake = 2, kUnitStar = 3 };

// Integrate blocks: kIntegrateUnits units per block, their atoms staged in a
// shared-memory table of at most kIntegrateTable entries.
constexpr int kIntegrateUnits = 32;
constexpr int kIntegrateTable = kIntegrateUnits * kMaxClusterAtoms;

// One integration unit: a free atom, a SETTLE water, or a SHAKE cluster.
struct UnitDev {
  int kind;
  int sys;
  int na;
  int nc;
  int base;                     // first entry of the unit's atoms in its block's table
  int atom[kMaxClusterAtoms];   // global atom indices
  float dist[kMaxClusterConstraints];
  unsigned char ci[kMaxClusterConstraints];
  unsigned char cj[kMaxClusterConstraints];
};

// Per-system constants, uploaded once (and again by setBox).
struct SysDev {
  int n_atoms, atom_off;
  int n_slots, slot_off;  // n_slots is a multiple of 32
  int n_blocks, block_off;
  int n_cells, cell_off;
  int cdim[3];
  int tile_off, tile_cap;
  int triclinic;
  int energy_base;
  // box, row-major a b c, reduced form; inverse M with f = r . M (M[v*3+u])
  float box_f[9];
  float min_width;   // narrowest perpendicular width of the cell, nm
  float inv_f[9];
  long long box_fx[9];  // lattice vectors, 2^32 fixed point
  long long inv_fx[9];  // M, 2^32 fixed point (fold and cells)
  // pair coordinates
  int pc_shift;
  float pc_inv;      // 2^-pc_shift
  float cut2u;       // cut2 in pair-coordinate units, cut2 2^(2 pc_shift)
  int pc_box[9];     // lattice in pair-coordinate units
  int pc_half[3];    // half of the diagonal in pair-coordinate units
  float pc_inv_diag[3];  // 1/diagonal in pair-coordinate units
  float cut2, list2, half_skin2, alpha, alpha_2_sqrtpi;
  float gauss_scale;  // -alpha^2 log2(e): exp(-(alpha r)^2) = 2^(r^2 gauss_scale)
  // the inner list: tiles with a pair inside (cutoff + inner skin)^2, re-pruned
  // from the outer list once an atom has moved (inner skin / 2)^2 since the last prune
  float inner2, half_inner2;
  // the inner prune also tests tiles flagged for per-pair images: worth it in
  // small cells, where nearly every tile is, and not where only a few are
  int prune_per_pair;
  // PME
  int grid[3];
  int kzh;            // Kz/2 + 1
  long long grid_off;   // real grids (int64 charge, f32 potential)
  long long cgrid_off;  // complex half spectrum
  int mod_off;          // moduli: x at mod_off, y at +Kx, z at +Kx+Ky
  int tw_off[3];        // twiddle tables per axis
  int radices[3][kMaxRadices];
  int nradix[3];
  long long umat[6];  // K o M, 2^32 fixed: u_a = x m0 + y m1 + z m2, u_b = y m3 + z m4, u_c = z m5
  float umat_f[9];    // K o M as f32, [v*3+u]
  float pme_pref;     // ONE_4PI_EPS0 * 2 pi / V
  float exp_scale;    // -1 / (4 alpha^2)
  // integrator
  int unit_off, n_units;
  int iblk_off, n_iblk;
  int com_freq;
  double total_mass;
};

// Run options shared by every system of an engine (src/gpu/integrate.ts:170).
struct RunDev {
  float dt, velocity_scale, noise_scale, kt;
  float tolerance;
  unsigned int seed;
  int integrator;
  int draw_noise;
  int always_rebuild;
};

// ---------------------------------------------------------- fixed point --
// 64-bit fixed point at 2^32 (src/gpu/kernels/fixed64.wgsl:7-21).  A native
// int64 makes the two-word carry arithmetic of the reference unnecessary, and
// `__float2ll_rn(x * 2^32)` is exactly its round-half-even magnitude
// decomposition: scaling by 2^32 is exact and ties keep their parity.
__device__ __forceinline__ long long to_fixed(float x) { return __float2ll_rn(x * 4294967296.0f); }
__device__ __forceinline__ float from_fixed(long long v) {
  return __ll2float_rn(v) * 2.3283064365386963e-10f;
}
__device__ __forceinline__ void add_fixed(unsigned long long* slot, float x) {
  atomicAdd(slot, static_cast<unsigned long long>(to_fixed(x)));
}
__device__ __forceinline__ void add_fixed64(unsigned long long* slot, long long v) {
  atomicAdd(slot, static_cast<unsigned long long>(v));
}

// ---------------------------------------------------- pair coordinates --
// A 2^32 fixed-point coordinate as int32 at 2^shift per nm, rounded.
__device__ __forceinline__ int to_pair_coordinate(long long v, int shift) {
  const int down = 32 - shift;
  return static_cast<int>((v + (1ll << (down - 1))) >> down);
}

// The lattice translation a rebuild stored for a slot: three signed 10-bit
// counts in one word.
__device__ __forceinline__ void unpack_fold(int w, long long& na, long long& nb, long long& nc) {
  na = (w << 22) >> 22;
  nb = (w << 12) >> 22;
  nc = (w << 2) >> 22;
}

// The pair coordinates of a position folded by (na, nb, nc) lattice vectors.
// The list kernel writes them at a rebuild or a prune and the integrator after
// every step, through this one function, so both give the same bits.
__device__ __forceinline__ int4 pair_coordinate(const SysDev& S, long long x, long long y, long long z, long long na,
                                                long long nb, long long nc) {
  x -= na * S.box_fx[0] + nb * S.box_fx[3] + nc * S.box_fx[6];
  y -= nb * S.box_fx[4] + nc * S.box_fx[7];
  z -= nc * S.box_fx[8];
  return make_int4(to_pair_coordinate(x, S.pc_shift), to_pair_coordinate(y, S.pc_shift),
                   to_pair_coordinate(z, S.pc_shift), 0);
}

// ------------------------------------------------------------------ RNG --
// Threefry-2x32-20 and Box-Muller, the device twin of src/reference/random.ts
// (random.wgsl:30-83).  The integer part is bit-exact with the oracle.
constexpr unsigned int kThermostatDomain = 0x9e3779b9u;

__device__ __forceinline__ uint2 threefry2x32(uint2 ctr, uint2 key) {
  const unsigned int ks2 = 0x1bd11bdau ^ key.x ^ key.y;
  const unsigned int ks[3] = {key.x, key.y, ks2};
  unsigned int x0 = ctr.x + key.x, x1 = ctr.y + key.y;
  const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
#pragma unroll
  for (int r = 0; r < 20; ++r) {
    x0 += x1;
    x1 = __funnelshift_l(x1, x1, rot[r & 7]) ^ x0;
    if ((r & 3) == 3) {
      const unsigned int inj = (r + 1) >> 2;
      x0 += ks[inj % 3];
      x1 += ks[(inj + 1) % 3] + inj;
    }
  }
  return make_uint2(x0, x1);
}

__device__ __forceinline__ float open_unit(unsigned int bits) {
  return (float(bits >> 9) + 0.5f) * 1.1920928955078125e-7f;
}

__device__ __forceinline__ float2 normal_pair(uint2 ctr, uint2 key) {
  const uint2 b = threefry2x32(ctr, key);
  const float radius = sqrtf(-2.0f * logf(open_unit(b.x)));
  float s, c;
  sincospif(2.0f * open_unit(b.y), &s, &c);
  return make_float2(radius * c, radius * s);
}

// ------------------------------------------------------------- helpers ---
__device__ __forceinline__ int find_system(const int* prefix, int count, int index) {
  int lo = 0, hi = count;  // prefix[count] is the total
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= index) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The interaction-mask bits of row l of tile ti (one bit per j): a word per
// row for 32x32 tiles, a byte per row (four to a word) for 8x8 tiles.
template <int C>
__device__ __forceinline__ unsigned int row_bits(const unsigned int* masks, long long ti, int l) {
  if (C == 32) return masks[ti * 32 + l];
  return (masks[ti * (C * C / 32) + (l >> 2)] >> ((l & 3) * 8)) & 0xFFu;
}

// A tile's lattice image, kept beside its shift in the tile's int4 (w): bit
// 0 asks for the per-pair minimum image, bits 1-30 hold the image's lattice
// counts (three signed 10-bit values), from which the shift in pair-coordinate
// units follows for any box -- so a small box change (a barostat move) can
// keep the list and recompute the shifts.
__host__ __device__ __forceinline__ int tile_flags(bool per_pair, int na, int nb, int nc) {
  return (per_pair ? 1 : 0) | ((na & 1023) << 1) | ((nb & 1023) << 11) | ((nc & 1023) << 21);
}
__device__ __forceinline__ bool tile_per_pair(int w) { return (w & 1) != 0; }
__device__ __forceinline__ int4 tile_shift_for(const SysDev& S, int w) {
  const int na = (w << 21) >> 22, nb = (w << 11) >> 22, nc = (w << 1) >> 22;
  const unsigned sx = unsigned(na) * unsigned(S.pc_box[0]) + unsigned(nb) * unsigned(S.pc_box[3]) +
                      unsigned(nc) * unsigned(S.pc_box[6]);
  const unsigned sy = unsigned(nb) * unsigned(S.pc_box[4]) + unsigned(nc) * unsigned(S.pc_box[7]);
  const unsigned sz = unsigned(nc) * unsigned(S.pc_box[8]);
  return make_int4(int(sx), int(sy), int(sz), w);
}

// Minimum image of a pair-coordinate difference (int32 at 2^pc_shift per nm).
template <bool TRICLINIC>
__device__ __forceinline__ void min_image(const SysDev& S, int& dx, int& dy, int& dz) {
  if (!TRICLINIC) {
    if (dx > S.pc_half[0]) dx -= S.pc_box[0];
    if (dx < -S.pc_half[0]) dx += S.pc_box[0];
    if (dy > S.pc_half[1]) dy -= S.pc_box[4];
    if (dy < -S.pc_half[1]) dy += S.pc_box[4];
    if (dz > S.pc_half[2]) dz -= S.pc_box[8];
    if (dz < -S.pc_half[2]) dz += S.pc_box[8];
  } else {
    // Sequential reduction against c, b, a (nonbonded.ts:241), the count
    // estimated in f32 and applied in integers.
    const int kc = __float2int_rn(dz * S.pc_inv_diag[2]);
    dz -= kc * S.pc_box[8];
    dy -= kc * S.pc_box[7];
    dx -= kc * S.pc_box[6];
    const int kb = __float2int_rn(dy * S.pc_inv_diag[1]);
    dy -= kb * S.pc_box[4];
    dx -= kb * S.pc_box[3];
    const int ka = __float2int_rn(dx * S.pc_inv_diag[0]);
    dx -= ka * S.pc_box[0];
  }
}

// u = r . M on the mesh, exactly in 2^32 fixed point, for the spline argument
// of the PME spread and gather.  r is the 2^32 fixed-point position.
__device__ __forceinline__ long long fixed_mul(long long a, long long b) {
  const __int128 p = static_cast<__int128>(a) * static_cast<__int128>(b);
  return static_cast<long long>(p >> 32);
}

}  // namespace mdb
