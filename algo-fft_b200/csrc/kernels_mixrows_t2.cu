// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_2(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 5>, 64, 3, 0>,
                              MixCfg<MixSched<10, 5>, 64, 2, 0>>());  // 50
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 7>, 64, 2, 0>,
                              MixCfg<MixSched<9, 7>, 32, 2, 9>>());  // 63
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 5>, 64, 2, 0>,
                              MixCfg<MixSched<15, 5>, 32, 3, 0>>());  // 75
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 9>, 32, 3, 10>,
                              MixCfg<MixSched<10, 9>, 32, 2, 10>>());  // 90
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 7>, 64, 1, 0>,
                              MixCfg<MixSched<15, 7>, 32, 1, 0>>());  // 105
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 5>, 64, 2, 0>,
                              MixCfg<MixSched<25, 5>, 32, 2, 0>>());  // 125
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 10>, 32, 2, 0>,
                              MixCfg<MixSched<14, 10>, 16, 2, 14>>());  // 140
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 10>, 32, 2, 0>,
                              MixCfg<MixSched<16, 10>, 16, 2, 16>>());  // 160
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 12>, 32, 1, 15>,
                              MixCfg<MixSched<15, 12>, 16, 2, 15>>());  // 180
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 10>, 32, 2, 0>,
                              MixCfg<MixSched<20, 10>, 16, 2, 0>>());  // 200
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15>, 32, 1, 0>,
                              MixCfg<MixSched<15, 15>, 16, 2, 0>>());  // 225
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 10>, 32, 2, 0>,
                              MixCfg<MixSched<25, 10>, 16, 2, 0>>());  // 250
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 14>, 16, 3, 0>,
                              MixCfg<MixSched<20, 14>, 8, 2, 20>>());  // 280
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 15>, 16, 2, 0>,
                              MixCfg<MixSched<21, 15>, 8, 2, 21>>());  // 315
  v.push_back(mix_rows_entry<MixCfg<MixSched<49, 7>, 16, 3, 0>,
                              MixCfg<MixSched<49, 7>, 8, 3, 0>>());  // 343
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 18>, 16, 2, 21>,
                              MixCfg<MixSched<21, 18>, 8, 2, 21>>());  // 378
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 15>, 16, 2, 0>,
                              MixCfg<MixSched<27, 15>, 8, 2, 0>>());  // 405
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 16>, 16, 2, 0>,
                              MixCfg<MixSched<28, 16>, 8, 2, 0>>());  // 448
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 14>, 16, 2, 0>,
                              MixCfg<MixSched<35, 14>, 8, 1, 0>>());  // 490
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 21>, 8, 3, 25>,
                              MixCfg<MixSched<25, 21>, 4, 3, 25>>());  // 525
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 24>, 8, 3, 0>,
                              MixCfg<MixSched<24, 24>, 4, 4, 0>>());  // 576
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 21>, 8, 2, 30>,
                              MixCfg<MixSched<30, 21>, 4, 2, 30>>());  // 630
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 25>, 8, 3, 27>,
                              MixCfg<MixSched<27, 25>, 4, 2, 27>>());  // 675
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 27>, 8, 3, 0>,
                              MixCfg<MixSched<27, 27>, 4, 2, 0>>());  // 729
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 24>, 8, 2, 0>,
                              MixCfg<MixSched<32, 24>, 4, 2, 32>>());  // 768
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 28>, 8, 2, 30>,
                              MixCfg<MixSched<30, 28>, 4, 2, 30>>());  // 840
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 28>, 8, 2, 32>,
                              MixCfg<MixSched<32, 28>, 4, 2, 32>>());  // 896
  v.push_back(mix_rows_entry<MixCfg<MixSched<36, 27>, 8, 2, 36>,
                              MixCfg<MixSched<36, 27>, 4, 1, 0>>());  // 972
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 32>, 4, 4, 0>,
                              MixCfg<MixSched<32, 32>, 2, 4, 0>>());  // 1024
}

}  // namespace gfft
