// k_barostat.cu -- the Monte Carlo volume move's position update on the device.
//
// src/reference/barostat.ts:210 (`scaleMolecules`, loop.ts:602-641): every
// molecule's centre (the plain mean of its atoms' positions) moves by the box
// scale; the atoms keep their offsets from it.  The reference reads the
// positions back to the host and writes the trial positions again; here one
// thread per molecule backs the positions up and moves them in place, and a
// rejected move restores the backup, so a volume move never copies
// coordinates across PCIe.
#include "device_state.h"

namespace mdb {
namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_scale_molecules(Dev d, int first_mol, int n_mol, double scale) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n_mol; m += gridDim.x * blockDim.x) {
    const int lo = d.mol_off[first_mol + m], hi = d.mol_off[first_mol + m + 1];
    double c[3] = {0, 0, 0};
    for (int k = lo; k < hi; ++k) {
      const int a = d.mol_atoms[k];
      d.bx[a] = d.px[a];
      d.by[a] = d.py[a];
      d.bz[a] = d.pz[a];
      c[0] += static_cast<double>(d.px[a]) * 2.3283064365386963e-10;
      c[1] += static_cast<double>(d.py[a]) * 2.3283064365386963e-10;
      c[2] += static_cast<double>(d.pz[a]) * 2.3283064365386963e-10;
    }
    double off[3];
    for (int k = 0; k < 3; ++k) {
      const double mean = c[k] / double(hi - lo);
      off[k] = scale * mean - mean;
    }
    for (int k = lo; k < hi; ++k) {
      const int a = d.mol_atoms[k];
      d.px[a] = __double2ll_rn((static_cast<double>(d.px[a]) * 2.3283064365386963e-10 + off[0]) * 4294967296.0);
      d.py[a] = __double2ll_rn((static_cast<double>(d.py[a]) * 2.3283064365386963e-10 + off[1]) * 4294967296.0);
      d.pz[a] = __double2ll_rn((static_cast<double>(d.pz[a]) * 2.3283064365386963e-10 + off[2]) * 4294967296.0);
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_restore_positions(Dev d, int atom_off, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = atom_off + i;
    d.px[a] = d.bx[a];
    d.py[a] = d.by[a];
    d.pz[a] = d.bz[a];
  }
}

// Sum over the molecules of one system of (r_i - R) (x) F_i, R the plain mean
// of the molecule's positions and F_i the total force on atom i (slot order,
// int64 fixed point): the difference between the atomic and the molecular
// virial.  FP64, one thread per molecule, fixed-order block partials.
__global__ void __launch_bounds__(kThreads) k_molecular_offsets(Dev d, int first_mol, int n_mol, int slot_off,
                                                                  double* partials) {
  __shared__ double red[9][kThreads / 32];
  double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n_mol; m += gridDim.x * blockDim.x) {
    const int lo = d.mol_off[first_mol + m], hi = d.mol_off[first_mol + m + 1];
    double c[3] = {0, 0, 0};
    for (int k = lo; k < hi; ++k) {
      const int a = d.mol_atoms[k];
      c[0] += static_cast<double>(d.px[a]);
      c[1] += static_cast<double>(d.py[a]);
      c[2] += static_cast<double>(d.pz[a]);
    }
    for (int k = 0; k < 3; ++k) c[k] /= double(hi - lo);
    for (int k = lo; k < hi; ++k) {
      const int a = d.mol_atoms[k];
      const int gs = slot_off + d.rank[a];
      const double r[3] = {(static_cast<double>(d.px[a]) - c[0]) * 2.3283064365386963e-10,
                           (static_cast<double>(d.py[a]) - c[1]) * 2.3283064365386963e-10,
                           (static_cast<double>(d.pz[a]) - c[2]) * 2.3283064365386963e-10};
      const double f[3] = {static_cast<double>(static_cast<long long>(d.fx[gs])) * 2.3283064365386963e-10,
                           static_cast<double>(static_cast<long long>(d.fy[gs])) * 2.3283064365386963e-10,
                           static_cast<double>(static_cast<long long>(d.fz[gs])) * 2.3283064365386963e-10};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) w[3 * i + j] += r[i] * f[j];
    }
  }
  for (int c = 0; c < 9; ++c) {
    double v = w[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double t = 0;
    for (int k = 0; k < kThreads / 32; ++k) t += red[threadIdx.x][k];
    partials[blockIdx.x * 9 + threadIdx.x] = t;
  }
}

// After the box of system s changed by a small amount (a volume move or its
// undo, positions scaled or restored): its slots' pair coordinates from the
// new positions under the list's folds, its tiles' shifts from their lattice
// counts and the new box, and the integrator's displacement tests -- half the
// skin from the list's reference positions, half the inner skin from the last
// prune's -- which here ask the list kernels for a rebuild or a prune
// directly.  So the list survives the move unless an atom went too far.
__global__ void __launch_bounds__(kThreads) k_after_box_change(Dev d, int s) {
  const SysDev& S = d.sys[s];
  const int n_tiles = min(d.tile_count[s], S.tile_cap);
  const int n_inner = d.inner ? min(d.in_count[s], S.tile_cap) : 0;
  const int n = max(S.n_slots, max(n_tiles, n_inner));
  bool moved = false, strayed = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < S.n_slots) {
      const int gs = S.slot_off + i;
      const int a = d.order[gs];
      if (a >= 0) {
        const long long x = d.px[a], y = d.py[a], z = d.pz[a];
        long long na, nb, nc;
        unpack_fold(d.fold[gs], na, nb, nc);
        d.pc[gs] = pair_coordinate(S, x, y, z, na, nb, nc);
        const float ex = from_fixed(x - d.refx[a]), ey = from_fixed(y - d.refy[a]), ez = from_fixed(z - d.refz[a]);
        moved |= ex * ex + ey * ey + ez * ez > S.half_skin2;
        if (d.inner) {
          const float qx = from_fixed(x - d.prx[a]), qy = from_fixed(y - d.pry[a]), qz = from_fixed(z - d.prz[a]);
          strayed |= qx * qx + qy * qy + qz * qz > S.half_inner2;
        }
      }
    }
    if (i < n_tiles) {
      const long long t = static_cast<long long>(S.tile_off) + i;
      d.tile_shift[t] = tile_shift_for(S, d.tile_shift[t].w);
    }
    if (i < n_inner) {
      const long long t = static_cast<long long>(S.tile_off) + i;
      d.in_shift[t] = tile_shift_for(S, d.in_shift[t].w);
    }
  }
  if (moved) {
    atomicExch(&d.rebuild_now[s], 1);
    atomicExch(d.any_rebuild, 1);
  }
  if (strayed) {
    atomicExch(&d.prune_now[s], 1);
    atomicExch(d.any_prune, 1);
  }
}

int blocks_for(int n) { return std::max(1, std::min((n + kThreads - 1) / kThreads, 148 * 8)); }

}  // namespace

void launch_scale_molecules(const Dev& d, int first_mol, int n_mol, double scale, cudaStream_t st) {
  k_scale_molecules<<<blocks_for(n_mol), kThreads, 0, st>>>(d, first_mol, n_mol, scale);
}

int molecular_offset_blocks(int n_mol) { return std::max(1, std::min((n_mol + kThreads - 1) / kThreads, 148)); }

void launch_molecular_offsets(const Dev& d, int first_mol, int n_mol, int slot_off, double* partials,
                              cudaStream_t st) {
  k_molecular_offsets<<<molecular_offset_blocks(n_mol), kThreads, 0, st>>>(d, first_mol, n_mol, slot_off, partials);
}

void launch_after_box_change(const Dev& d, int s, int n_slots, int tile_cap, cudaStream_t st) {
  k_after_box_change<<<blocks_for(std::max(n_slots, tile_cap)), kThreads, 0, st>>>(d, s);
}

void launch_restore_positions(const Dev& d, int atom_off, int n, cudaStream_t st) {
  k_restore_positions<<<blocks_for(n), kThreads, 0, st>>>(d, atom_off, n);
}

}  // namespace mdb
