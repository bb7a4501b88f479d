// pb_carp_blocks.hpp -- block colouring of the rows for the CARP sweep
// (host code, no CUDA).
//
// A Kaczmarz projection of row i reads and writes X at the columns of row i
// and at i itself (the shift term).  Rows are grouped into blocks of nearby
// rows; a block's footprint is the union of those index sets.  Blocks whose
// footprints are disjoint do not interact, so the blocks are coloured such
// that blocks of one colour have disjoint footprints, and a sweep runs colour
// by colour with one thread block per block: it stages the footprint rows of
// X in shared memory, projects its rows there and writes the footprint back.
// X is then read and written about once per sweep (times the footprint
// overhead) instead of once per colour of a row colouring.
//
// Inside a block the rows are ordered in steps: rows of one step have
// pairwise disjoint index sets (a distance-2 colouring of the block's rows),
// so a step runs in parallel and the steps run one after another.  The sweep
// therefore equals the sequential Kaczmarz sweep over the rows in the order
//   colour 0: step 0 of every block of colour 0, step 1 of every block, ...
//   colour 1: ...
// and every (colour, step) segment of that order is a distance-2 independent
// set of rows.  The backward sweep runs the same order reversed (colours and
// steps descending), as the builtin sweep reverses its row loop
// (kacz_loop_seq_def.h, backward branch).
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef __CUDACC__
#define PB_HD __host__ __device__
#else
#define PB_HD
#endif

namespace pb {

// One row block of the block-coloured sweep is one byte segment that the
// thread block copies to shared memory; segment b starts at b * stride
// (stride: the largest segment, a multiple of 16), so its address needs no
// lookup:
//   header     int32 nrows, nfp, nnz, nsteps
//   fp         int32 [nfp]       global X rows of the footprint, the block's
//                                own rows first (slots 0..nrows-1)
//   val        T [nnz]           entries, rows in block order
//   nd         T [2 nrows]       per row (sum_k a_ik^2, a_ii)
//   lcol       uint16 [nnz]      footprint slot of each entry's column
//   lrp        uint16 [nrows+1]  entry offsets of the rows
//   step       uint16 [nsteps+1] first row of each step
// each part starting on a 16-byte boundary.  Header and footprint rows come
// first: the X gather needs only them (carp_seg_head bytes).
PB_HD inline int carp_r16b(int x) { return (x + 15) & ~15; }

struct CarpSeg {
  int nrows, nfp, nnz, nsteps;
  int fp, val, nd, lcol, lrp, step, bytes;  // byte offsets inside the segment, size
};
PB_HD inline CarpSeg carp_seg(int nrows, int nfp, int nnz, int nsteps, int tsize)
{
  CarpSeg g;
  g.nrows = nrows;
  g.nfp = nfp;
  g.nnz = nnz;
  g.nsteps = nsteps;
  int o = 16;
  g.fp = o;
  o += carp_r16b(4 * nfp);
  g.val = o;
  o += carp_r16b(tsize * nnz);
  g.nd = o;
  o += carp_r16b(2 * tsize * nrows);
  g.lcol = o;
  o += carp_r16b(2 * nnz);
  g.lrp = o;
  o += carp_r16b(2 * (nrows + 1));
  g.step = o;
  o += carp_r16b(2 * (nsteps + 1));
  g.bytes = o;
  return g;
}
// bytes of header and footprint rows for footprints of at most max_fp rows
PB_HD inline int carp_seg_head(int max_fp) { return 16 + carp_r16b(4 * max_fp); }

// Shared-memory layout of the block sweep kernel (byte offsets): the X
// footprint rows (TPR slots of tsize bytes per row; a second set for the
// imaginary part), the block's rows of B and its segment (seg_stride bytes).
struct CarpSmem {
  int xs, xis, bs;
  int xbase, mbase, total;
};
PB_HD inline CarpSmem carp_smem_layout(int max_fp, int max_rows, int seg_stride, int tpr, int tsize, bool rc,
                                       bool hasb)
{
  CarpSmem L;
  int o = 0;
  L.xs = o;
  o += carp_r16b(max_fp * tpr * tsize);
  L.xis = o;
  if (rc) o += carp_r16b(max_fp * tpr * tsize);
  L.bs = o;
  if (hasb) o += carp_r16b(max_rows * tpr * tsize);
  L.xbase = 0;
  L.mbase = o;
  L.total = o + carp_r16b(seg_stride);
  return L;
}

struct CarpBlocks {
  int64_t nblocks = 0;
  int ncolors = 0;                     // block colours
  int max_rows = 0, max_fp = 0, max_nnz = 0, max_steps = 0;
  std::vector<int64_t> color_ptr;      // blocks [color_ptr[c], color_ptr[c+1]) have colour c
  std::vector<int64_t> row_ptr;        // rows of block b: [row_ptr[b], row_ptr[b+1]) of `rows`
  std::vector<int32_t> rows;           // block order: per block its rows, step by step
  std::vector<int64_t> fp_ptr;         // footprint of block b: fp[fp_ptr[b] .. fp_ptr[b+1])
  std::vector<int32_t> fp;             // global X rows; the block's own rows first, in `rows` order
  std::vector<int64_t> step_ptr;       // step starts of block b: step[step_ptr[b] .. step_ptr[b+1]]
  std::vector<uint16_t> step;          // local row offsets, nsteps+1 per block
  // sequential equivalent: rows sorted by (colour, step), with segment pointers
  std::vector<int32_t> seq_rows;
  std::vector<int64_t> seq_ptr;
};

// Grow blocks by breadth-first search over the row graph (row i is adjacent
// to the rows indexed by its columns and to the rows that hold column i),
// starting next to the blocks built so far (else at the lowest unassigned
// row); a row joins while the block has fewer than max_rows rows, its
// footprint stays within max_fp entries and its pattern within max_nnz
// entries.  Returns false when some single row has more than max_fp pattern
// entries (dense rows: use the row colouring).  prp/pcol is the pattern of
// the square matrix with every diagonal present; max_fp <= max_nnz.
inline bool carp_block_partition(int64_t n, const std::vector<int64_t>& prp, const std::vector<int32_t>& pcol,
                                 int max_rows, int max_fp, int max_nnz, CarpBlocks& B)
{
  if (max_fp > max_nnz) return false;
  for (int64_t i = 0; i < n; i++)
    if (prp[i + 1] - prp[i] > max_fp) return false;
  // transpose pattern: rows holding column c
  std::vector<int64_t> tp(n + 1, 0);
  for (int64_t p = 0; p < prp[n]; p++) tp[pcol[p] + 1]++;
  for (int64_t j = 0; j < n; j++) tp[j + 1] += tp[j];
  std::vector<int32_t> trow(prp[n]);
  {
    std::vector<int64_t> fill(tp.begin(), tp.end() - 1);
    for (int64_t i = 0; i < n; i++)
      for (int64_t p = prp[i]; p < prp[i + 1]; p++) trow[fill[pcol[p]]++] = (int32_t)i;
  }
  std::vector<int32_t> blk(n, -1);       // block of each row
  std::vector<int64_t> fpmark(n, -1);    // fpmark[c] == b: column c in the footprint of block b
  std::vector<int64_t> qmark(n, -1);     // qmark[r] == b: row r queued for block b
  std::vector<int32_t> queue, members, fpl;
  std::vector<int32_t> border;           // block-level BFS frontier: rows next to finished blocks
  B.row_ptr.assign(1, 0);
  B.fp_ptr.assign(1, 0);
  B.rows.clear();
  B.fp.clear();
  int64_t seed_scan = 0;
  size_t border_head = 0;
  int64_t nb = 0;
  int64_t assigned = 0;
  while (assigned < n) {
    // seed: a row next to an earlier block (keeps blocks compact and
    // adjacent), else the lowest unassigned row
    int32_t seed = -1;
    while (border_head < border.size()) {
      const int32_t r = border[border_head++];
      if (blk[r] < 0) { seed = r; break; }
    }
    if (seed < 0) {
      while (blk[seed_scan] >= 0) seed_scan++;
      seed = (int32_t)seed_scan;
    }
    queue.clear();
    members.clear();
    fpl.clear();
    queue.push_back(seed);
    qmark[seed] = nb;
    size_t head = 0;
    int64_t bnnz = 0;
    while (head < queue.size() && (int)members.size() < max_rows) {
      const int32_t r = queue[head++];
      // footprint growth if r joins (the seed always joins: its own pattern
      // fits both limits)
      int add = 0;
      for (int64_t p = prp[r]; p < prp[r + 1]; p++) add += fpmark[pcol[p]] != nb;
      if ((int)fpl.size() + add > max_fp || bnnz + (prp[r + 1] - prp[r]) > max_nnz) continue;
      bnnz += prp[r + 1] - prp[r];
      members.push_back(r);
      blk[r] = (int32_t)nb;
      for (int64_t p = prp[r]; p < prp[r + 1]; p++) {
        const int32_t c = pcol[p];
        if (fpmark[c] != nb) { fpmark[c] = nb; fpl.push_back(c); }
      }
      auto visit = [&](int32_t k) {
        if (blk[k] < 0 && qmark[k] != nb) { qmark[k] = nb; queue.push_back(k); }
      };
      for (int64_t p = prp[r]; p < prp[r + 1]; p++) visit(pcol[p]);
      for (int64_t t = tp[r]; t < tp[r + 1]; t++) visit(trow[t]);
    }
    // rows queued but not taken seed the next blocks
    for (size_t k = head; k < queue.size(); k++) border.push_back(queue[k]);
    for (size_t k = 0; k < head; k++)
      if (blk[queue[k]] < 0) border.push_back(queue[k]);
    assigned += (int64_t)members.size();
    // footprint: own rows first, then the other columns in first-touch order
    for (int32_t r : members) B.rows.push_back(r);
    for (int32_t r : members) B.fp.push_back(r);
    for (int32_t c : fpl)
      if (blk[c] != nb) B.fp.push_back(c);
    B.row_ptr.push_back((int64_t)B.rows.size());
    B.fp_ptr.push_back((int64_t)B.fp.size());
    nb++;
  }
  B.nblocks = nb;
  return true;
}

// Colour the blocks so that blocks of one colour have disjoint footprints
// (greedy in block order), then reorder blocks by colour, and order the rows
// of each block in steps (greedy distance-2 colouring inside the block, rows
// in their block order).  Fills the sequential row order with its
// (colour, step) segments.
inline bool carp_block_color(int64_t n, const std::vector<int64_t>& prp, const std::vector<int32_t>& pcol,
                             CarpBlocks& B)
{
  const int64_t nb = B.nblocks;
  // column -> blocks whose footprint holds it
  std::vector<int64_t> cp(n + 1, 0);
  for (int64_t b = 0; b < nb; b++)
    for (int64_t k = B.fp_ptr[b]; k < B.fp_ptr[b + 1]; k++) cp[B.fp[k] + 1]++;
  for (int64_t c = 0; c < n; c++) cp[c + 1] += cp[c];
  std::vector<int32_t> cblk(cp[n]);
  {
    std::vector<int64_t> fill(cp.begin(), cp.end() - 1);
    for (int64_t b = 0; b < nb; b++)
      for (int64_t k = B.fp_ptr[b]; k < B.fp_ptr[b + 1]; k++) cblk[fill[B.fp[k]]++] = (int32_t)b;
  }
  // conflict lists: blocks whose footprints meet
  std::vector<int64_t> ap(nb + 1, 0);
  std::vector<int32_t> adj;
  {
    std::vector<int64_t> seen(nb, -1);
    for (int64_t b = 0; b < nb; b++) {
      for (int64_t k = B.fp_ptr[b]; k < B.fp_ptr[b + 1]; k++) {
        const int32_t c = B.fp[k];
        for (int64_t t = cp[c]; t < cp[c + 1]; t++) {
          const int32_t o = cblk[t];
          if (o != b && seen[o] != b) {
            seen[o] = b;
            adj.push_back(o);
          }
        }
      }
      ap[b + 1] = (int64_t)adj.size();
    }
  }
  // greedy colouring in a given block order, then iterated greedy (blocks
  // visited colour class by colour class, classes in reverse order): never
  // more colours, often fewer, i.e. fewer launches per sweep
  std::vector<int64_t> mark;
  auto greedy = [&](const std::vector<int32_t>& ord, std::vector<int32_t>& col) {
    col.assign(nb, -1);
    mark.assign(mark.size(), -1);
    int nc = 0;
    for (int64_t k = 0; k < nb; k++) {
      const int64_t b = ord.empty() ? k : ord[k];
      for (int64_t t = ap[b]; t < ap[b + 1]; t++) {
        const int32_t co = col[adj[t]];
        if (co >= 0) {
          if ((int)mark.size() <= co) mark.resize(co + 1, -1);
          mark[co] = b;
        }
      }
      int c = 0;
      while (c < (int)mark.size() && mark[c] == b) c++;
      col[b] = c;
      nc = std::max(nc, c + 1);
    }
    return nc;
  };
  std::vector<int32_t> color, cand, vis(nb);
  int ncolor = greedy(std::vector<int32_t>(), color);
  for (int round = 0; round < 8 && ncolor > 1; round++) {
    std::vector<int64_t> start(ncolor + 1, 0);
    for (int64_t b = 0; b < nb; b++) start[ncolor - color[b]]++;
    for (int c = 0; c < ncolor; c++) start[c + 1] += start[c];
    for (int64_t b = 0; b < nb; b++) vis[start[ncolor - 1 - color[b]]++] = (int32_t)b;
    const int nc = greedy(vis, cand);
    if (nc > ncolor) break;
    color.swap(cand);
    ncolor = nc;
  }
  // blocks in colour order (stable)
  std::vector<int64_t> order(nb);
  {
    std::vector<int64_t> cnt(ncolor + 1, 0);
    for (int64_t b = 0; b < nb; b++) cnt[color[b] + 1]++;
    for (int c = 0; c < ncolor; c++) cnt[c + 1] += cnt[c];
    B.color_ptr = cnt;
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t b = 0; b < nb; b++) order[fill[color[b]]++] = b;
  }
  // steps inside every block; per footprint slot a mask of the steps that
  // touch it
  CarpBlocks R;
  R.nblocks = nb;
  R.ncolors = ncolor;
  R.color_ptr = B.color_ptr;
  R.row_ptr.assign(1, 0);
  R.fp_ptr.assign(1, 0);
  R.step_ptr.assign(1, 0);
  std::vector<int32_t> slot(n, -1);
  std::vector<uint64_t> used;
  std::vector<int> rstep;
  std::vector<int32_t> brows;
  for (int c = 0; c < ncolor; c++) {
    std::vector<std::vector<int32_t>> cs;  // rows of colour c by step
    for (int64_t k = B.color_ptr[c]; k < B.color_ptr[c + 1]; k++) {
      const int64_t b = order[k];
      const int64_t r0 = B.row_ptr[b], r1 = B.row_ptr[b + 1];
      const int64_t f0 = B.fp_ptr[b], f1 = B.fp_ptr[b + 1];
      const int nr = (int)(r1 - r0), nf = (int)(f1 - f0);
      for (int64_t s = f0; s < f1; s++) slot[B.fp[s]] = (int32_t)(s - f0);
      used.assign(nf, 0);
      rstep.assign(nr, 0);
      int nsteps = 0;
      for (int q = 0; q < nr; q++) {
        const int32_t r = B.rows[r0 + q];
        uint64_t forb = 0;
        for (int64_t p = prp[r]; p < prp[r + 1]; p++) forb |= used[slot[pcol[p]]];
        if (~forb == 0) return false;  // more than 64 steps
        int s = 0;
        while (forb >> s & 1) s++;
        rstep[q] = s;
        for (int64_t p = prp[r]; p < prp[r + 1]; p++) used[slot[pcol[p]]] |= uint64_t(1) << s;
        nsteps = std::max(nsteps, s + 1);
      }
      // rows by step (stable), footprint: own rows in that order, then the rest
      brows.clear();
      std::vector<uint16_t> st(nsteps + 1, 0);
      for (int q = 0; q < nr; q++) st[rstep[q] + 1]++;
      for (int s = 0; s < nsteps; s++) st[s + 1] += st[s];
      brows.resize(nr);
      {
        std::vector<uint16_t> fill(st.begin(), st.end() - 1);
        for (int q = 0; q < nr; q++) brows[fill[rstep[q]]++] = B.rows[r0 + q];
      }
      if ((int)cs.size() < nsteps) cs.resize(nsteps);
      for (int s = 0; s < nsteps; s++)
        for (int q = st[s]; q < st[s + 1]; q++) cs[s].push_back(brows[q]);
      for (int32_t r : brows) R.rows.push_back(r);
      for (int32_t r : brows) R.fp.push_back(r);
      for (int64_t s = f0 + nr; s < f1; s++) R.fp.push_back(B.fp[s]);
      for (uint16_t v : st) R.step.push_back(v);
      R.row_ptr.push_back((int64_t)R.rows.size());
      R.fp_ptr.push_back((int64_t)R.fp.size());
      R.step_ptr.push_back((int64_t)R.step.size());
      R.max_rows = std::max(R.max_rows, nr);
      R.max_fp = std::max(R.max_fp, nf);
      R.max_steps = std::max(R.max_steps, nsteps);
      int64_t nz = 0;
      for (int q = 0; q < nr; q++) nz += prp[B.rows[r0 + q] + 1] - prp[B.rows[r0 + q]];
      R.max_nnz = std::max<int64_t>(R.max_nnz, nz);
      for (int64_t s = f0; s < f1; s++) slot[B.fp[s]] = -1;
    }
    for (auto& v : cs) {
      R.seq_ptr.push_back((int64_t)R.seq_rows.size());
      for (int32_t r : v) R.seq_rows.push_back(r);
    }
  }
  R.seq_ptr.push_back((int64_t)R.seq_rows.size());
  B = std::move(R);
  return true;
}

// Device array of the block-coloured sweep, built from the blocks and the
// CRS matrix (rp, col, val; n square): the segments (layout above) at a
// fixed stride.
template <class T>
struct CarpBlockLayout {
  std::vector<unsigned char> seg;
  int stride = 0;
};

template <class T>
void carp_block_layout(const CarpBlocks& B, int64_t n, const int64_t* rp, const int32_t* col, const T* val,
                       CarpBlockLayout<T>& L)
{
  const int64_t nb = B.nblocks;
  std::vector<CarpSeg> gs(nb);
  L.stride = 16;
  for (int64_t b = 0; b < nb; b++) {
    const int64_t r0 = B.row_ptr[b], r1 = B.row_ptr[b + 1];
    int nz = 0;
    for (int64_t q = r0; q < r1; q++) nz += (int)(rp[B.rows[q] + 1] - rp[B.rows[q]]);
    gs[b] = carp_seg((int)(r1 - r0), (int)(B.fp_ptr[b + 1] - B.fp_ptr[b]), nz,
                     (int)(B.step_ptr[b + 1] - B.step_ptr[b] - 1), (int)sizeof(T));
    L.stride = std::max(L.stride, gs[b].bytes);
  }
  L.seg.assign((size_t)nb * L.stride, 0);
  std::vector<int32_t> slot(n, -1);
  for (int64_t b = 0; b < nb; b++) {
    const int64_t r0 = B.row_ptr[b], r1 = B.row_ptr[b + 1];
    const int64_t f0 = B.fp_ptr[b], f1 = B.fp_ptr[b + 1];
    const int64_t s0 = B.step_ptr[b], s1 = B.step_ptr[b + 1];
    const CarpSeg& g = gs[b];
    unsigned char* p = L.seg.data() + (size_t)b * L.stride;
    const int32_t hdr[4] = {g.nrows, g.nfp, g.nnz, g.nsteps};
    memcpy(p, hdr, sizeof(hdr));
    int32_t* fp = (int32_t*)(p + g.fp);
    T* v = (T*)(p + g.val);
    T* nd = (T*)(p + g.nd);
    uint16_t* lc = (uint16_t*)(p + g.lcol);
    uint16_t* lr = (uint16_t*)(p + g.lrp);
    uint16_t* st = (uint16_t*)(p + g.step);
    for (int64_t k = f0; k < f1; k++) {
      slot[B.fp[k]] = (int32_t)(k - f0);
      fp[k - f0] = B.fp[k];
    }
    int e = 0;
    lr[0] = 0;
    for (int64_t q = r0; q < r1; q++) {
      const int64_t i = B.rows[q];
      T sq = T(0), dg = T(0);
      for (int64_t k = rp[i]; k < rp[i + 1]; k++) {
        v[e] = val[k];
        lc[e] = (uint16_t)slot[col[k]];
        e++;
        sq += val[k] * val[k];
        if (col[k] == i) dg = val[k];
      }
      lr[q - r0 + 1] = (uint16_t)e;
      nd[2 * (q - r0)] = sq;
      nd[2 * (q - r0) + 1] = dg;
    }
    for (int64_t k = s0; k < s1; k++) st[k - s0] = B.step[k];
    for (int64_t k = f0; k < f1; k++) slot[B.fp[k]] = -1;
  }
}

}  // namespace pb
