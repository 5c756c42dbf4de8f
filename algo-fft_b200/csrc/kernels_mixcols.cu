// The compiled mixed-radix column tiles (gfft_mixcols.cuh) of every 7-smooth
// column length 48..1024: the table the generated kernels_mixcols_t*.cu files
// fill, and the launcher the four-step and column-batch plans call.
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

}  // namespace

bool mix_cols_supported(int64_t L) { return find(L) != nullptr; }

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
