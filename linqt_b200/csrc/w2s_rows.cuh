// Row arithmetic of the supercell builder (supercell.cu), shared by its kernels: pure
// functions of the plan tables, usable from host code as well.
#pragma once

#include "w2s.cuh"

#define LQ_HD __host__ __device__

namespace linqt {
namespace w2s {

struct PlanView {
  int wbb, dx, dy, dz, K;
  int nz, ny, nx;  // runs per level, all groups
  long ncells, n;
  const int *grp_key0, *grp_z0, *kz, *ky, *kx, *kleaf, *ko1, *kgrp;
  const Node *zn, *yn, *xn;
  const double2 *kval;
  const int4 *kpack;
  const int *kgo;
};

template <class T>
LQ_HD inline T ld(const T *p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}

LQ_HD inline int first_at_least(const Node *nd, int lo, int hi, int t) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld(&nd[mid].val) < t)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// offset of run idx in its parent's column order when runs [k, end) wrap to the front
LQ_HD inline int rotated(const Node *nd, int idx, int k, int end, int total) {
  const int pk = k < end ? ld(&nd[k].pre) : total;
  const int pi = ld(&nd[idx].pre);
  return idx >= k ? pi - pk : total - pk + pi;
}

LQ_HD inline Node load_node(const Node *nd, int i) {
  Node r;
  r.val = ld(&nd[i].val);
  r.pre = ld(&nd[i].pre);
  r.size = ld(&nd[i].size);
  r.c0 = ld(&nd[i].c0);
  r.nc = ld(&nd[i].nc);
  r.par = ld(&nd[i].par);
  return r;
}

// keys of group g whose column in cell (sx, sy, sz) lies left of the diagonal: the runs
// that wrap at each level, then the cell's own position one level down, then the own
// cell's orbitals below g
LQ_HD inline int keys_below(const PlanView &p, int g, int sx, int sy, int sz) {
  const int ng = ld(&p.grp_key0[g + 1]) - ld(&p.grp_key0[g]);
  if (ng == 0) return 0;
  const int z0 = ld(&p.grp_z0[g]), z1 = ld(&p.grp_z0[g + 1]);
  int k = first_at_least(p.zn, z0, z1, p.dz - sz);
  int w = ng - (k < z1 ? ld(&p.zn[k].pre) : ng);
  const Node Z = load_node(p.zn, z0);
  if (Z.val != 0) return w;
  k = first_at_least(p.yn, Z.c0, Z.c0 + Z.nc, p.dy - sy);
  w += Z.size - (k < Z.c0 + Z.nc ? ld(&p.yn[k].pre) : Z.size);
  const Node Y = load_node(p.yn, Z.c0);
  if (Y.val != 0) return w;
  k = first_at_least(p.xn, Y.c0, Y.c0 + Y.nc, p.dx - sx);
  w += Y.size - (k < Y.c0 + Y.nc ? ld(&p.xn[k].pre) : Y.size);
  const Node X = load_node(p.xn, Y.c0);
  if (X.val != 0) return w;
  int lo = X.c0, hi = X.c0 + X.size;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld(&p.ko1[mid]) < g)
      lo = mid + 1;
    else
      hi = mid;
  }
  return w + (lo - X.c0);
}

LQ_HD inline void cell_coords(const PlanView &p, long s, int &sx, int &sy, int &sz) {
  const unsigned us = (unsigned)s;  // ncells < 2^31
  const unsigned q = us / (unsigned)p.dx;
  sx = (int)(us - q * (unsigned)p.dx);
  const unsigned q2 = q / (unsigned)p.dy;
  sy = (int)(q - q2 * (unsigned)p.dy);
  sz = (int)q2;
}

LQ_HD inline int row_count(const PlanView &p, long r) {
  const unsigned ur = (unsigned)r;  // n < 2^31
  const unsigned s = ur / (unsigned)p.wbb;
  const int g = (int)(ur - s * (unsigned)p.wbb);
  int sx, sy, sz;
  cell_coords(p, s, sx, sy, sz);
  return ld(&p.grp_key0[g + 1]) - ld(&p.grp_key0[g]) - keys_below(p, g, sx, sy, sz);
}


// entry of key t in cell s: false when it lies in the lower triangle, else its position in
// the output and its column.  rowptr holds the row offsets.
LQ_HD inline bool item_entry(const PlanView &p, const int *rowptr, long s, int t, long &pos, long &col) {
  const int g = ld(&p.kgrp[t]);
  const long r = s * p.wbb + g;
  const int rp0 = ld(&rowptr[r]);
  const int ng = ld(&p.grp_key0[g + 1]) - ld(&p.grp_key0[g]);
  const int below = ng - (ld(&rowptr[r + 1]) - rp0);
  int sx, sy, sz;
  cell_coords(p, s, sx, sy, sz);
  const int zi = ld(&p.kz[t]), yi = ld(&p.ky[t]), xi = ld(&p.kx[t]);
  const int z0 = ld(&p.grp_z0[g]), z1 = ld(&p.grp_z0[g + 1]);
  int rank = rotated(p.zn, zi, first_at_least(p.zn, z0, z1, p.dz - sz), z1, ng);
  const Node Z = load_node(p.zn, zi);
  rank += rotated(p.yn, yi, first_at_least(p.yn, Z.c0, Z.c0 + Z.nc, p.dy - sy), Z.c0 + Z.nc, Z.size);
  const Node Y = load_node(p.yn, yi);
  rank += rotated(p.xn, xi, first_at_least(p.xn, Y.c0, Y.c0 + Y.nc, p.dx - sx), Y.c0 + Y.nc, Y.size);
  rank += ld(&p.kleaf[t]);
  if (rank < below) return false;
  int cz = Z.val + sz, cy = Y.val + sy, cx = ld(&p.xn[xi].val) + sx;
  if (cz >= p.dz) cz -= p.dz;
  if (cy >= p.dy) cy -= p.dy;
  if (cx >= p.dx) cx -= p.dx;
  col = (((long)cz * p.dy + cy) * p.dx + cx) * p.wbb + ld(&p.ko1[t]);
  pos = (long)rp0 + rank - below;
  return true;
}

// Per-cell table of the cell-blocked fill (k_fill_cells): for cell s
//   [0, nz)                 rotated offset of every z run inside its group
//   [nz, nz+ny)             ... of every y run inside its z run
//   [nz+ny, nz+ny+nx)       ... of every x run inside its y run
//   [nz+ny+nx, nz+ny+2nx)   target cell of every x run
//   then wbb first stored positions and wbb below-diagonal counts of the cell's rows
// so that a key's place is four table reads and its leaf index.
LQ_HD inline int cell_table_size(const PlanView &p) { return p.nz + p.ny + 2 * p.nx + 2 * p.wbb; }
LQ_HD inline int cell_table_items(const PlanView &p) { return p.nz + p.ny + p.nx + p.wbb; }

LQ_HD inline void cell_table_entry(const PlanView &p, long s, int sx, int sy, int sz, int j, const int *rowptr,
                                   int *tab) {
  if (j < p.nz) {
    const int g = ld(&p.zn[j].par);
    const int z0 = ld(&p.grp_z0[g]), z1 = ld(&p.grp_z0[g + 1]);
    const int ng = ld(&p.grp_key0[g + 1]) - ld(&p.grp_key0[g]);
    tab[j] = rotated(p.zn, j, first_at_least(p.zn, z0, z1, p.dz - sz), z1, ng);
    return;
  }
  j -= p.nz;
  if (j < p.ny) {
    const Node Z = load_node(p.zn, ld(&p.yn[j].par));
    tab[p.nz + j] = rotated(p.yn, j, first_at_least(p.yn, Z.c0, Z.c0 + Z.nc, p.dy - sy), Z.c0 + Z.nc, Z.size);
    return;
  }
  j -= p.ny;
  if (j < p.nx) {
    const Node Y = load_node(p.yn, ld(&p.xn[j].par));
    tab[p.nz + p.ny + j] = rotated(p.xn, j, first_at_least(p.xn, Y.c0, Y.c0 + Y.nc, p.dx - sx), Y.c0 + Y.nc, Y.size);
    int cz = ld(&p.zn[Y.par].val) + sz, cy = Y.val + sy, cx = ld(&p.xn[j].val) + sx;
    if (cz >= p.dz) cz -= p.dz;
    if (cy >= p.dy) cy -= p.dy;
    if (cx >= p.dx) cx -= p.dx;
    tab[p.nz + p.ny + p.nx + j] = (int)(((long)cz * p.dy + cy) * p.dx + cx);
    return;
  }
  j -= p.nx;  // row (s, j)
  const long r = s * p.wbb + j;
  const int rp0 = ld(&rowptr[r]);
  const int ng = ld(&p.grp_key0[j + 1]) - ld(&p.grp_key0[j]);
  const int base = p.nz + p.ny + 2 * p.nx;
  tab[base + j] = rp0;
  tab[base + p.wbb + j] = ng - (ld(&rowptr[r + 1]) - rp0);
}

// key k (packed runs and leaf, group << 16 | target orbital) in the cell whose table is tab:
// false in the lower triangle, else output place and column
LQ_HD inline bool key_place(const PlanView &p, int4 k, int go, const int *tab, long &pos, long &col) {
  const int g = go >> 16, o1 = go & 0xffff;
  const int rank = tab[k.x] + tab[p.nz + k.y] + tab[p.nz + p.ny + k.z] + k.w;
  const int base = p.nz + p.ny + 2 * p.nx;
  const int below = tab[base + p.wbb + g];
  if (rank < below) return false;
  pos = (long)tab[base + g] + rank - below;
  col = (long)tab[p.nz + p.ny + p.nx + k.z] * p.wbb + o1;
  return true;
}

LQ_HD inline bool key_entry(const PlanView &p, int t, const int *tab, long &pos, long &col) {
  return key_place(p, ld(&p.kpack[t]), ld(&p.kgo[t]), tab, pos, col);
}

}  // namespace w2s
}  // namespace linqt
