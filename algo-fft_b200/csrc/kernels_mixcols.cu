// The compiled mixed-radix column tiles (gfft_mixcols.cuh) of every 7-smooth
// column length 48..1024 and the Bluestein chain's passes on them
// (gfft_mixbs.cuh): the tables the generated kernels_mixcols_t*.cu and
// kernels_mixbs_t*.cu files fill, and the launchers the plans call.
#include <algorithm>
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_0(std::vector<MixEntry>& v);
void mix_part_1(std::vector<MixEntry>& v);
void mix_part_2(std::vector<MixEntry>& v);
void mix_part_3(std::vector<MixEntry>& v);
void mix_part_4(std::vector<MixEntry>& v);
void mix_part_5(std::vector<MixEntry>& v);
void mix_part_6(std::vector<MixEntry>& v);
void mix_part_7(std::vector<MixEntry>& v);
void mix_rows_part_0(std::vector<MixRowsEntry>& v);
void mix_rows_part_1(std::vector<MixRowsEntry>& v);
void mix_rows_part_2(std::vector<MixRowsEntry>& v);
void mix_rows_part_3(std::vector<MixRowsEntry>& v);
void mix_rows_part_4(std::vector<MixRowsEntry>& v);
void mix_rows_part_5(std::vector<MixRowsEntry>& v);
void mix_rows_part_6(std::vector<MixRowsEntry>& v);
void mix_rows_part_7(std::vector<MixRowsEntry>& v);
void mix_bs_part_0(std::vector<MixBsEntry>& v);
void mix_bs_part_1(std::vector<MixBsEntry>& v);
void mix_bs_part_2(std::vector<MixBsEntry>& v);

namespace {

const std::vector<MixEntry>& table() {
  static const std::vector<MixEntry> t = [] {
    std::vector<MixEntry> v;
    for (auto part : {&mix_part_0, &mix_part_1, &mix_part_2, &mix_part_3, &mix_part_4, &mix_part_5, &mix_part_6,
                      &mix_part_7})
      part(v);
    std::sort(v.begin(), v.end(), [](const MixEntry& a, const MixEntry& b) { return a.L < b.L; });
    return v;
  }();
  return t;
}

const MixEntry* find(int64_t L) {
  const std::vector<MixEntry>& t = table();
  auto it = std::lower_bound(t.begin(), t.end(), L, [](const MixEntry& e, int64_t l) { return e.L < l; });
  return it != t.end() && it->L == L ? &*it : nullptr;
}

const std::vector<MixRowsEntry>& rows_table() {
  static const std::vector<MixRowsEntry> t = [] {
    std::vector<MixRowsEntry> v;
    for (auto part : {&mix_rows_part_0, &mix_rows_part_1, &mix_rows_part_2, &mix_rows_part_3, &mix_rows_part_4,
                      &mix_rows_part_5, &mix_rows_part_6, &mix_rows_part_7})
      part(v);
    std::sort(v.begin(), v.end(), [](const MixRowsEntry& a, const MixRowsEntry& b) { return a.L < b.L; });
    return v;
  }();
  return t;
}

const MixRowsEntry* rows_find(int64_t L) {
  for (const MixRowsEntry& e : rows_table())
    if (e.L == L) return &e;
  return nullptr;
}

const std::vector<MixBsEntry>& bs_table() {
  static const std::vector<MixBsEntry> t = [] {
    std::vector<MixBsEntry> v;
    for (auto part : {&mix_bs_part_0, &mix_bs_part_1, &mix_bs_part_2}) part(v);
    std::sort(v.begin(), v.end(), [](const MixBsEntry& a, const MixBsEntry& b) { return a.L < b.L; });
    return v;
  }();
  return t;
}

const MixBsEntry* bs_find(int64_t L) {
  for (const MixBsEntry& e : bs_table())
    if (e.L == L) return &e;
  return nullptr;
}

}  // namespace

bool mix_cols_supported(int64_t L) { return find(L) != nullptr; }

int64_t bs_mixed_length(int64_t n, int64_t* m1) {
  int64_t best = 0, a_best = 0;
  const std::vector<MixBsEntry>& t = bs_table();
  for (size_t i = 0; i < t.size(); ++i)
    for (size_t j = i; j < t.size(); ++j) {
      const int64_t a = t[i].L, b = t[j].L, m = a * b;
      if (m < 2 * n - 1) continue;
      // the smallest M; among equal ones the most balanced split
      if (best == 0 || m < best || (m == best && a > a_best)) {
        best = m;
        a_best = a;
      }
    }
  if (m1) *m1 = a_best;
  return best;
}

bool mix_rows_supported(int prec, int64_t L) {
  const MixRowsEntry* e = rows_find(L);
  return e && (prec == kC64 || prec == kC128) && e->fn[prec][0];
}

cudaError_t exec_mix_rows(int prec, int dir, int64_t L, const MixRowsParams& p, cudaStream_t st) {
  if (!mix_rows_supported(prec, L)) return cudaErrorNotSupported;
  return rows_find(L)->fn[prec][dir < 0 ? 0 : 1](p, st);
}

int mix_bs_width(int prec, int64_t L) {
  const MixBsEntry* e = bs_find(L);
  return e && (prec == kC64 || prec == kC128) ? e->nc[prec] : 0;
}

cudaError_t exec_mix_bs(int prec, int kind, int64_t L, MixBsParams p, int64_t count, cudaStream_t st) {
  const MixBsEntry* e = bs_find(L);
  if (!e || kind < BSK_IN || kind > BSK_OUT || (prec != kC64 && prec != kC128)) return cudaErrorNotSupported;
  int64_t blocks = count;  // item mode: CTAs
  if (!p.items) {
    const int nc = e->nc[prec];
    p.tiles = (p.M / L + nc - 1) / nc;
    blocks = p.tiles * count;
  }
  return e->fn[prec][kind](p, blocks, st);
}

std::vector<int64_t> mix_cols_lengths() {
  std::vector<int64_t> v;
  for (const MixEntry& e : table()) v.push_back(e.L);
  return v;
}

int mix_cols_width(int prec, int pass, int64_t L) {
  const MixEntry* e = find(L);
  if (!e || (prec != kC64 && prec != kC128)) return 0;
  return pass == MIX_PASS1 ? e->nc[prec] : e->nc2[prec];
}

cudaError_t exec_mix_cols(int prec, int dir, int pass, int64_t L, MixColsParams p, int64_t count, cudaStream_t st) {
  const MixEntry* e = find(L);
  if (!e || (pass != MIX_PASS1 && pass != MIX_PASS2) || (prec != kC64 && prec != kC128)) return cudaErrorNotSupported;
  if (p.items) {
    p.tiles = count;  // item mode: `count` CTAs, each finds its transform
    count = 1;
  } else {
    const int nc = pass == MIX_PASS1 ? e->nc[prec] : e->nc2[prec];
    p.tiles = (p.ncols + nc - 1) / nc;
  }
  return e->fn[prec][dir < 0 ? 0 : 1][pass - 1](p, count, st);
}

}  // namespace gfft
