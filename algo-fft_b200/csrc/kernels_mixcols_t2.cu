// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_2(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<10, 5>, 16, 8, 0>,
                         MixCfg<MixSched<10, 5>, 16, 8, 0>,
                         MixCfg<MixSched<10, 5>, 8, 8, 0>,
                         MixCfg<MixSched<10, 5>, 8, 8, 0>>());  // 50
  v.push_back(mix_entry<MixCfg<MixSched<15, 5>, 16, 8, 0>,
                         MixCfg<MixSched<15, 5>, 16, 8, 0>,
                         MixCfg<MixSched<15, 5>, 8, 8, 0>,
                         MixCfg<MixSched<15, 5>, 8, 8, 0>>());  // 75
  v.push_back(mix_entry<MixCfg<MixSched<15, 7>, 16, 6, 0>,
                         MixCfg<MixSched<15, 7>, 16, 6, 0>,
                         MixCfg<MixSched<15, 7>, 8, 6, 0>,
                         MixCfg<MixSched<15, 7>, 8, 6, 0>>());  // 105
  v.push_back(mix_entry<MixCfg<MixSched<14, 10>, 16, 5, 0>,
                         MixCfg<MixSched<14, 10>, 16, 5, 0>,
                         MixCfg<MixSched<14, 10>, 8, 4, 14>,
                         MixCfg<MixSched<14, 10>, 8, 4, 14>>());  // 140
  v.push_back(mix_entry<MixCfg<MixSched<15, 12>, 16, 3, 15>,
                         MixCfg<MixSched<15, 12>, 16, 3, 15>,
                         MixCfg<MixSched<15, 12>, 8, 4, 15>,
                         MixCfg<MixSched<15, 12>, 8, 4, 15>>());  // 180
  v.push_back(mix_entry<MixCfg<MixSched<15, 15>, 16, 3, 0>,
                         MixCfg<MixSched<15, 15>, 16, 3, 0>,
                         MixCfg<MixSched<15, 15>, 8, 4, 0>,
                         MixCfg<MixSched<15, 15>, 8, 4, 0>>());  // 225
  v.push_back(mix_entry<MixCfg<MixSched<20, 14>, 16, 3, 0>,
                         MixCfg<MixSched<20, 14>, 16, 3, 0>,
                         MixCfg<MixSched<20, 14>, 8, 2, 20>,
                         MixCfg<MixSched<20, 14>, 8, 2, 20>>());  // 280
  v.push_back(mix_entry<MixCfg<MixSched<49, 7>, 16, 3, 0>,
                         MixCfg<MixSched<49, 7>, 16, 3, 0>,
                         MixCfg<MixSched<49, 7>, 8, 3, 0>,
                         MixCfg<MixSched<49, 7>, 8, 3, 0>>());  // 343
  v.push_back(mix_entry<MixCfg<MixSched<27, 15>, 16, 2, 0>,
                         MixCfg<MixSched<27, 15>, 16, 2, 0>,
                         MixCfg<MixSched<27, 15>, 8, 2, 0>,
                         MixCfg<MixSched<27, 15>, 8, 2, 0>>());  // 405
  v.push_back(mix_entry<MixCfg<MixSched<35, 14>, 16, 2, 0>,
                         MixCfg<MixSched<35, 14>, 16, 2, 0>,
                         MixCfg<MixSched<35, 14>, 8, 1, 0>,
                         MixCfg<MixSched<35, 14>, 8, 1, 0>>());  // 490
  v.push_back(mix_entry<MixCfg<MixSched<24, 24>, 8, 3, 0>,
                         MixCfg<MixSched<24, 24>, 8, 3, 0>,
                         MixCfg<MixSched<24, 24>, 4, 4, 0>,
                         MixCfg<MixSched<24, 24>, 4, 4, 0>>());  // 576
  v.push_back(mix_entry<MixCfg<MixSched<27, 25>, 8, 3, 27>,
                         MixCfg<MixSched<27, 25>, 8, 3, 27>,
                         MixCfg<MixSched<27, 25>, 4, 2, 27>,
                         MixCfg<MixSched<27, 25>, 4, 2, 27>>());  // 675
  v.push_back(mix_entry<MixCfg<MixSched<32, 24>, 8, 2, 0>,
                         MixCfg<MixSched<32, 24>, 8, 2, 0>,
                         MixCfg<MixSched<32, 24>, 4, 2, 32>,
                         MixCfg<MixSched<12, 8, 8>, 4, 3, 0>>());  // 768
  v.push_back(mix_entry<MixCfg<MixSched<32, 28>, 8, 2, 32>,
                         MixCfg<MixSched<32, 28>, 8, 2, 32>,
                         MixCfg<MixSched<32, 28>, 4, 2, 32>,
                         MixCfg<MixSched<32, 28>, 4, 2, 32>>());  // 896
  v.push_back(mix_entry<MixCfg<MixSched<32, 32>, 8, 2, 0>,
                         MixCfg<MixSched<32, 32>, 8, 2, 0>,
                         MixCfg<MixSched<32, 32>, 4, 2, 0>,
                         MixCfg<MixSched<32, 32>, 4, 2, 0>>());  // 1024
}

}  // namespace gfft
