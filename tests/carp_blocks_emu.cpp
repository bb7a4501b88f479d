// Host emulation of the block-coloured CARP sweep (k_kacz_blocks in
// phist_b200/csrc/pb_carp.cuh) for the CPU tests: builds the blocks and the
// device layout with the library's own host code (pb_carp_blocks.hpp), then
// runs the kernel's schedule -- colour launches, one thread block per row
// block: the segment head, then the rest of the segment with the X and B
// rows, the steps and the write-back -- on the host with every index
// checked against the arrays and shared-memory regions it addresses:
//   * every copy stays inside its source array and its shared region;
//   * footprint rows are valid rows of X, and blocks of one launch have
//     disjoint footprints;
//   * step bounds, entry offsets and footprint-local columns stay inside the
//     block, and the rows of one step touch disjoint footprint slots.
// Any violation exits with status 3 and a message.
//
// usage: carp_blocks_emu <in> <out> <max_rows> <max_fp> <max_nnz> <wide>
//   wide 1: X and B copied in 16-byte pieces (when the column count is even)
//   in : int64 n, nnz, nv, has_b; int64 rp[n+1]; int32 col[nnz];
//        f64 val[nnz], shifts[nv], omega[nv], b[n*nv] (if has_b), x[n*nv]
//   out: int64 ok (0: no block layout), nseg; int32 rows[n];
//        int64 seg_ptr[nseg+1]; f64 x[n*nv];
//        int64 nblocks, ncolors, max_fp, max_rows, seg_stride, max_steps,
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
  if (argc != 7) {
    fprintf(stderr, "usage: %s in out max_rows max_fp max_nnz wide\n", argv[0]);
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
  // X and B pieces: 2 doubles (16 bytes) when the columns fill whole pieces
  const int W = (atoi(argv[6]) != 0 && nv % 2 == 0) ? 2 : 1;
  const int PW = TPR / W;
  const CarpSmem S = carp_smem_layout(B.max_fp, B.max_rows, L.stride, TPR, 8, false, hasb);
  const int head = carp_seg_head(B.max_fp);
  EMU_CHECK(S.mbase % 16 == 0 && S.bs % 16 == 0 && L.stride % 16 == 0);
  EMU_CHECK(head <= L.stride && (int64_t)L.seg.size() == B.nblocks * (int64_t)L.stride);
  std::vector<unsigned char> smem(S.total);
  std::vector<int64_t> owner(n, -1);
  int64_t launch_id = 0;

  // the thread block of row block blk
  auto run_block = [&](int64_t blk, int dir) {
    memset(smem.data(), 0xff, smem.size());
    unsigned char* mb = smem.data() + S.mbase;
    unsigned char* xb = smem.data() + S.xbase;
    const int64_t off = blk * (int64_t)L.stride;
    // H: header and footprint rows
    EMU_CHECK(off + head <= (int64_t)L.seg.size());
    EMU_CHECK(S.mbase + head <= S.total);
    memcpy(mb, L.seg.data() + off, head);
    // X: rest of the segment, X and B rows
    const int32_t* hdr = (const int32_t*)mb;
    const CarpSeg sg = carp_seg(hdr[0], hdr[1], hdr[2], hdr[3], 8);
    EMU_CHECK(sg.bytes % 16 == 0 && sg.bytes <= L.stride && S.mbase + sg.bytes <= S.total);
    if (sg.bytes > head) memcpy(mb + head, L.seg.data() + off + head, sg.bytes - head);
    EMU_CHECK(sg.nfp <= B.max_fp && sg.nrows <= B.max_rows && sg.nrows <= sg.nfp);
    const int32_t* fps = (const int32_t*)(mb + 16);
    double* xs = (double*)(xb + S.xs);
    double* bs = (double*)(xb + S.bs);
    for (int e = 0; e < sg.nfp * PW; e++) {
      const int u = e / PW, j = (e % PW) * W;
      if (j >= nv) continue;
      EMU_CHECK(16 + 4 * (u + 1) <= head);
      const int64_t g = fps[u];
      EMU_CHECK(g >= 0 && g < n);
      EMU_CHECK(S.xs + 8 * (u * TPR + j + W) <= S.xis);
      if (j == 0) {
        EMU_CHECK(owner[g] != launch_id);  // disjoint footprints in one launch
        owner[g] = launch_id;
      }
      for (int k = 0; k < W; k++) xs[u * TPR + j + k] = x[g * nv + j + k];
    }
    if (hasb)
      for (int e = 0; e < sg.nrows * PW; e++) {
        const int r = e / PW, j = (e % PW) * W;
        if (j >= nv) continue;
        EMU_CHECK(S.bs + 8 * (r * TPR + j + W) <= S.mbase);
        for (int k = 0; k < W; k++) bs[r * TPR + j + k] = b[(int64_t)fps[r] * nv + j + k];
      }
    const double* vs = (const double*)(mb + sg.val);
    const double* nds = (const double*)(mb + sg.nd);
    const uint16_t* lcs = (const uint16_t*)(mb + sg.lcol);
    const uint16_t* lrs = (const uint16_t*)(mb + sg.lrp);
    const uint16_t* sts = (const uint16_t*)(mb + sg.step);
    EMU_CHECK(sg.nsteps >= 1 && sg.nsteps <= 64 && sts[0] == 0 && sts[sg.nsteps] == sg.nrows);
    std::vector<int> touched(sg.nfp);
    auto step = [&](int st) {
      const int lo = sts[st], hi = sts[st + 1];
      EMU_CHECK(lo <= hi && hi <= sg.nrows);
      std::fill(touched.begin(), touched.end(), -1);
      for (int r = lo; r < hi; r++) {
        EMU_CHECK(lrs[r] <= lrs[r + 1] && lrs[r + 1] <= sg.nnz);
        auto touch = [&](int sl) {
          EMU_CHECK(sl >= 0 && sl < sg.nfp);
          EMU_CHECK(touched[sl] == -1 || touched[sl] == r);
          touched[sl] = r;
        };
        touch(r);
        for (int p = lrs[r]; p < lrs[r + 1]; p++) touch(lcs[p]);
      }
      for (int r = lo; r < hi; r++)
        for (int j = 0; j < nv; j++) {
          const double s_ = sr[j];
          double rn = nds[2 * r] - 2.0 * nds[2 * r + 1] * s_ + s_ * s_;
          if (rn == 0.0) rn = 1.0;
          const double f = om[j] / rn;
          double tr = -s_ * xs[r * TPR + j];
          for (int p = lrs[r]; p < lrs[r + 1]; p++) tr += vs[p] * xs[lcs[p] * TPR + j];
          if (hasb) tr -= bs[r * TPR + j];
          tr *= f;
          xs[r * TPR + j] += tr * s_;
          for (int p = lrs[r]; p < lrs[r + 1]; p++) xs[lcs[p] * TPR + j] -= tr * vs[p];
        }
    };
    if (dir & 1)
      for (int st = 0; st < sg.nsteps; st++) step(st);
    if (dir & 2)
      for (int st = sg.nsteps - 1; st >= 0; st--) step(st);
    for (int e = 0; e < sg.nfp * PW; e++) {
      const int u = e / PW, j = (e % PW) * W;
      if (j >= nv) continue;
      const int64_t g = fps[u];
      for (int k = 0; k < W; k++) x[g * nv + j + k] = xs[u * TPR + j + k];
    }
  };
  auto launch = [&](int c, int dir) {
    for (int64_t blk = B.color_ptr[c]; blk < B.color_ptr[c + 1]; blk++) run_block(blk, dir);
    launch_id++;
  };
  // forward over the colours, the last one forward and straight back, then
  // backward over the others
  const int C = B.ncolors;
  for (int c = 0; c < C - 1; c++) launch(c, 1);
  launch(C - 1, 3);
  for (int c = C - 2; c >= 0; c--) launch(c, 2);

  const int64_t ohead[2] = {1, (int64_t)B.seq_ptr.size() - 1};
  wr(fo, ohead, 2);
  wr(fo, B.seq_rows.data(), B.seq_rows.size());
  wr(fo, B.seq_ptr.data(), B.seq_ptr.size());
  wr(fo, x.data(), x.size());
  const int64_t st[8] = {B.nblocks, B.ncolors, B.max_fp, B.max_rows, L.stride, B.max_steps, S.total,
                         (int64_t)B.fp.size()};
  wr(fo, st, 8);
  fclose(fo);
  return 0;
}
