// Host emulation of the block-coloured CARP sweep (k_kacz_blocks in
// phist_b200/csrc/pb_carp.cuh) for the CPU tests: builds the blocks and the
// device layout with the library's own host code (pb_carp_blocks.hpp), then
// runs the kernel's schedule -- colour launches, one thread block per row
// block, its 16-byte segment copies, footprint gather, steps and write-back
// -- on the host with every index checked against the arrays and
// shared-memory regions it addresses:
//   * every segment copy stays inside its array and its shared region;
//   * footprint rows are valid rows of X, and blocks of one launch have
//     disjoint footprints;
//   * step bounds, entry offsets and footprint-local columns stay inside the
//     block, and the rows of one step touch disjoint footprint slots.
// Any violation exits with status 3 and a message.
//
// usage: carp_blocks_emu <in> <out> <max_rows> <max_fp> <max_nnz>
//   in : int64 n, nnz, nv, has_b; int64 rp[n+1]; int32 col[nnz];
//        f64 val[nnz], shifts[nv], omega[nv], b[n*nv] (if has_b), x[n*nv]
//   out: int64 ok (0: no block layout), nseg; int32 rows[n];
//        int64 seg_ptr[nseg+1]; f64 x[n*nv];
//        int64 nblocks, ncolors, max_fp, max_rows, max_nnz, max_steps,
//        smem_bytes, footprint_total
#include "../phist_b200/csrc/pb_carp_blocks.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace pb;

#define EMU_CHECK(c)                                               \
  do {                                                             \
    if (!(c)) {                                                    \
      fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
      exit(3);                                                     \
    }                                                              \
  } while (0)

template <class V>
static void rd(FILE* f, V* p, size_t n)
{
  if (n && fread(p, sizeof(V), n, f) != n) {
    fprintf(stderr, "short read\n");
    exit(2);
  }
}
template <class V>
static void wr(FILE* f, const V* p, size_t n)
{
  if (n) fwrite(p, sizeof(V), n, f);
}

int main(int argc, char** argv)
{
  if (argc != 6) {
    fprintf(stderr, "usage: %s in out max_rows max_fp max_nnz\n", argv[0]);
    return 2;
  }
  FILE* fi = fopen(argv[1], "rb");
  if (!fi) return 2;
  int64_t hdr[4];
  rd(fi, hdr, 4);
  const int64_t n = hdr[0], nnz = hdr[1];
  const int nv = (int)hdr[2];
  const bool hasb = hdr[3] != 0;
  std::vector<int64_t> rp(n + 1);
  std::vector<int32_t> col(nnz);
  std::vector<double> val(nnz), sr(nv), om(nv), b(hasb ? n * nv : 0), x(n * nv);
  rd(fi, rp.data(), n + 1);
  rd(fi, col.data(), nnz);
  rd(fi, val.data(), nnz);
  rd(fi, sr.data(), nv);
  rd(fi, om.data(), nv);
  rd(fi, b.data(), b.size());
  rd(fi, x.data(), x.size());
  fclose(fi);
  EMU_CHECK(nv >= 1 && nv <= 32);

  // pattern with every diagonal present, as carp_build forms it
  std::vector<int64_t> prp(n + 1, 0);
  std::vector<int32_t> pcol;
  for (int64_t i = 0; i < n; i++) {
    bool hd = false;
    for (int64_t p = rp[i]; p < rp[i + 1]; p++) {
      pcol.push_back(col[p]);
      hd |= col[p] == i;
    }
    if (!hd) pcol.push_back((int32_t)i);
    prp[i + 1] = (int64_t)pcol.size();
  }
  CarpBlocks B;
  const bool ok = n > 0 && carp_block_partition(n, prp, pcol, atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), B) &&
                  carp_block_color(n, prp, pcol, B);
  FILE* fo = fopen(argv[2], "wb");
  if (!fo) return 2;
  if (!ok) {
    const int64_t z[2] = {0, 0};
    wr(fo, z, 2);
    fclose(fo);
    return 0;
  }
  CarpBlockLayout<double> L;
  carp_block_layout<double>(B, n, rp.data(), col.data(), val.data(), L);
  EMU_CHECK(B.max_steps <= 64);
  const int TPR = nv <= 1 ? 1 : nv <= 2 ? 2 : nv <= 4 ? 4 : nv <= 8 ? 8 : nv <= 16 ? 16 : 32;
  const CarpSmem S = carp_smem_layout(B.max_fp, B.max_rows, L.max_nnz, TPR, 8, false, hasb);
  std::vector<unsigned char> smem(S.total);
  std::vector<int64_t> owner(n, -1);
  int64_t launch_id = 0;

  auto run_block = [&](int64_t blk, int dir) {
    const CarpBlockDesc d = L.desc[blk];
    EMU_CHECK(d.nfp <= B.max_fp && d.nrows <= B.max_rows && d.nnz <= L.max_nnz && d.nrows <= d.nfp);
    memset(smem.data(), 0xff, smem.size());
    auto seg = [&](const void* base, size_t bytes, int64_t off, int nchunks, int s0, int s1) {
      EMU_CHECK(off % 16 == 0);
      EMU_CHECK(off + 16 * (int64_t)nchunks <= (int64_t)bytes);
      EMU_CHECK(s0 + 16 * nchunks <= s1);
      memcpy(smem.data() + s0, (const char*)base + off, 16 * (size_t)nchunks);
    };
    seg(L.val.data(), L.val.size() * 8, d.ent * 8, carp_r8(d.nnz) * 8 / 16, S.val, S.nd);
    seg(L.lcol.data(), L.lcol.size() * 2, d.ent * 2, carp_r8(d.nnz) * 2 / 16, S.lcol, S.lrp);
    seg(L.lrp.data(), L.lrp.size() * 2, d.row * 2, carp_r8(d.nrows + 1) * 2 / 16, S.lrp, S.step);
    seg(L.nd.data(), L.nd.size() * 8, d.row * 16, carp_r8(d.nrows) * 2 * 8 / 16, S.nd, S.fp);
    seg(L.fp.data(), L.fp.size() * 4, d.fp * 4, ((d.nfp + 3) & ~3) * 4 / 16, S.fp, S.lcol);
    seg(L.step.data(), L.step.size() * 2, d.step * 2, carp_r8(d.nsteps + 1) * 2 / 16, S.step, S.total);
    double* xs = (double*)(smem.data() + S.xs);
    double* bs = (double*)(smem.data() + S.bs);
    const double* vs = (const double*)(smem.data() + S.val);
    const double* nds = (const double*)(smem.data() + S.nd);
    const int32_t* fps = (const int32_t*)(smem.data() + S.fp);
    const uint16_t* lcs = (const uint16_t*)(smem.data() + S.lcol);
    const uint16_t* lrs = (const uint16_t*)(smem.data() + S.lrp);
    const uint16_t* sts = (const uint16_t*)(smem.data() + S.step);
    for (int e = 0; e < d.nfp * TPR; e++) {
      const int u = e / TPR, j = e % TPR;
      if (j >= nv) continue;
      EMU_CHECK(d.fp + u < (int64_t)L.fp.size());
      const int64_t g = L.fp[d.fp + u];
      EMU_CHECK(g >= 0 && g < n);
      EMU_CHECK(S.xs + 8 * (e + 1) <= S.xis);
      if (j == 0) {
        EMU_CHECK(owner[g] != launch_id);  // disjoint footprints in one launch
        owner[g] = launch_id;
      }
      xs[e] = x[g * nv + j];
    }
    if (hasb)
      for (int e = 0; e < d.nrows * TPR; e++) {
        const int r = e / TPR, j = e % TPR;
        if (j >= nv) continue;
        EMU_CHECK(S.bs + 8 * (e + 1) <= S.val);
        bs[e] = b[(int64_t)L.fp[d.fp + r] * nv + j];
      }
    EMU_CHECK(d.nsteps >= 1 && d.nsteps <= 64 && sts[0] == 0 && sts[d.nsteps] == d.nrows);
    std::vector<int> touched(d.nfp);
    auto step = [&](int s) {
      const int lo = sts[s], hi = sts[s + 1];
      EMU_CHECK(lo <= hi && hi <= d.nrows);
      std::fill(touched.begin(), touched.end(), -1);
      for (int r = lo; r < hi; r++) {
        EMU_CHECK(lrs[r] <= lrs[r + 1] && lrs[r + 1] <= d.nnz);
        auto touch = [&](int sl) {
          EMU_CHECK(sl >= 0 && sl < d.nfp);
          EMU_CHECK(touched[sl] == -1 || touched[sl] == r);
          touched[sl] = r;
        };
        touch(r);
        for (int p = lrs[r]; p < lrs[r + 1]; p++) touch(lcs[p]);
      }
      for (int e = 0; e < (hi - lo) * TPR; e++) {
        const int r = lo + e / TPR, j = e % TPR;
        if (j >= nv) continue;
        const double s_ = sr[j];
        double tr = -s_ * xs[r * TPR + j];
        for (int p = lrs[r]; p < lrs[r + 1]; p++) tr += vs[p] * xs[lcs[p] * TPR + j];
        if (hasb) tr -= bs[r * TPR + j];
        double rn = nds[2 * r] - 2.0 * nds[2 * r + 1] * s_ + s_ * s_;
        if (rn == 0.0) rn = 1.0;
        tr *= om[j] / rn;
        xs[r * TPR + j] += tr * s_;
        for (int p = lrs[r]; p < lrs[r + 1]; p++) xs[lcs[p] * TPR + j] -= tr * vs[p];
      }
    };
    if (dir & 1)
      for (int s = 0; s < d.nsteps; s++) step(s);
    if (dir & 2)
      for (int s = d.nsteps - 1; s >= 0; s--) step(s);
    for (int e = 0; e < d.nfp * TPR; e++) {
      const int u = e / TPR, j = e % TPR;
      if (j >= nv) continue;
      const int64_t g = fps[u];
      EMU_CHECK(g == L.fp[d.fp + u]);
      x[g * nv + j] = xs[e];
    }
  };
  auto launch = [&](int c, int dir) {
    for (int64_t blk = B.color_ptr[c]; blk < B.color_ptr[c + 1]; blk++) run_block(blk, dir);
    launch_id++;
  };
  const int C = B.ncolors;
  for (int c = 0; c < C - 1; c++) launch(c, 1);
  launch(C - 1, 3);
  for (int c = C - 2; c >= 0; c--) launch(c, 2);

  const int64_t head[2] = {1, (int64_t)B.seq_ptr.size() - 1};
  wr(fo, head, 2);
  wr(fo, B.seq_rows.data(), B.seq_rows.size());
  wr(fo, B.seq_ptr.data(), B.seq_ptr.size());
  wr(fo, x.data(), x.size());
  const int64_t st[8] = {B.nblocks, B.ncolors, B.max_fp, B.max_rows, L.max_nnz, B.max_steps, S.total,
                         (int64_t)B.fp.size()};
  wr(fo, st, 8);
  fclose(fo);
  return 0;
}
