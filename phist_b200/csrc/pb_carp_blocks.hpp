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
#include <vector>

#ifdef __CUDACC__
#define PB_HD __host__ __device__
#else
#define PB_HD
#endif

namespace pb {

// one row block of the block-coloured sweep; every offset is a multiple of
// 16 bytes in its array and every per-block segment is padded to 16 bytes,
// so the thread block copies its segments in 16-byte pieces
struct CarpBlockDesc {
  int64_t fp;     // first footprint entry (int32 global X rows), multiple of 4
  int64_t ent;    // first matrix entry (values, uint16 footprint slots), multiple of 8
  int64_t row;    // first row slot (uint16 entry offsets: nrows+1; (norm, diagonal) pairs), multiple of 8
  int64_t step;   // first step start (uint16 local rows: nsteps+1), multiple of 8
  int32_t nrows, nfp, nnz, nsteps;
};

PB_HD inline int carp_r8(int x) { return (x + 7) & ~7; }
PB_HD inline int carp_r16b(int x) { return (x + 15) & ~15; }

// shared-memory layout of the block sweep kernel (byte offsets), sized for
// the largest block; TPR slots of tsize bytes per X row
struct CarpSmem {
  int xs, xis, bs, val, nd, fp, lcol, lrp, step, total;
};
PB_HD inline CarpSmem carp_smem_layout(int max_fp, int max_rows, int max_nnz, int tpr, int tsize, bool rc,
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
  L.val = o;
  o += carp_r16b(carp_r8(max_nnz) * tsize);
  L.nd = o;
  o += carp_r16b(2 * carp_r8(max_rows + 1) * tsize);
  L.fp = o;
  o += carp_r16b(4 * ((max_fp + 3) & ~3));
  L.lcol = o;
  o += carp_r16b(2 * carp_r8(max_nnz));
  L.lrp = o;
  o += carp_r16b(2 * carp_r8(max_rows + 1));
  L.step = o;
  o += 2 * carp_r8(64 + 1);
  L.total = o;
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
  std::vector<int32_t> color(nb, -1);
  std::vector<int64_t> mark;
  int ncolor = 0;
  for (int64_t b = 0; b < nb; b++) {
    for (int64_t k = B.fp_ptr[b]; k < B.fp_ptr[b + 1]; k++) {
      const int32_t c = B.fp[k];
      for (int64_t t = cp[c]; t < cp[c + 1]; t++) {
        const int32_t o = cblk[t];
        if (o != b && color[o] >= 0) {
          if ((int)mark.size() <= color[o]) mark.resize(color[o] + 1, -1);
          mark[color[o]] = b;
        }
      }
    }
    int c = 0;
    while (c < (int)mark.size() && mark[c] == b) c++;
    color[b] = c;
    ncolor = std::max(ncolor, c + 1);
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

// Device arrays of the block-coloured sweep, built from the blocks and the
// CRS matrix (rp, col, val; n square): per block its footprint rows, its
// entries with footprint-local columns (rows in block order, the block's own
// rows being footprint slots 0..nrows-1), per row the entry offsets and the
// pair (sum_k a_ik^2, a_ii), and the step starts.
template <class T>
struct CarpBlockLayout {
  std::vector<CarpBlockDesc> desc;
  std::vector<int32_t> fp;
  std::vector<T> val, nd;
  std::vector<uint16_t> lcol, lrp, step;
  int max_nnz = 0;
};

template <class T>
void carp_block_layout(const CarpBlocks& B, int64_t n, const int64_t* rp, const int32_t* col, const T* val,
                       CarpBlockLayout<T>& L)
{
  const int64_t nb = B.nblocks;
  L.desc.assign(nb, CarpBlockDesc());
  std::vector<int32_t> slot(n, -1);
  for (int64_t b = 0; b < nb; b++) {
    const int64_t r0 = B.row_ptr[b], r1 = B.row_ptr[b + 1];
    const int64_t f0 = B.fp_ptr[b], f1 = B.fp_ptr[b + 1];
    const int64_t s0 = B.step_ptr[b], s1 = B.step_ptr[b + 1];
    CarpBlockDesc& d = L.desc[b];
    d.nrows = (int32_t)(r1 - r0);
    d.nfp = (int32_t)(f1 - f0);
    d.nsteps = (int32_t)(s1 - s0 - 1);
    d.fp = (int64_t)L.fp.size();
    for (int64_t k = f0; k < f1; k++) {
      slot[B.fp[k]] = (int32_t)(k - f0);
      L.fp.push_back(B.fp[k]);
    }
    while (L.fp.size() % 4) L.fp.push_back(0);
    d.ent = (int64_t)L.val.size();
    d.row = (int64_t)L.lrp.size();
    L.lrp.push_back(0);
    for (int64_t q = r0; q < r1; q++) {
      const int64_t i = B.rows[q];
      T sq = T(0), dg = T(0);
      for (int64_t p = rp[i]; p < rp[i + 1]; p++) {
        L.val.push_back(val[p]);
        L.lcol.push_back((uint16_t)slot[col[p]]);
        sq += val[p] * val[p];
        if (col[p] == i) dg = val[p];
      }
      L.lrp.push_back((uint16_t)(L.val.size() - d.ent));
      L.nd.push_back(sq);
      L.nd.push_back(dg);
    }
    d.nnz = (int32_t)(L.val.size() - d.ent);
    L.max_nnz = std::max(L.max_nnz, (int)d.nnz);
    while (L.val.size() % 8) {
      L.val.push_back(T(0));
      L.lcol.push_back(0);
    }
    while (L.lrp.size() % 8) L.lrp.push_back(0);
    L.nd.resize(2 * L.lrp.size(), T(0));
    d.step = (int64_t)L.step.size();
    for (int64_t k = s0; k < s1; k++) L.step.push_back(B.step[k]);
    while (L.step.size() % 8) L.step.push_back(0);
    for (int64_t k = f0; k < f1; k++) slot[B.fp[k]] = -1;
  }
}

}  // namespace pb
