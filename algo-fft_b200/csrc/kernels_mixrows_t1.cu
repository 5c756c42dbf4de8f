// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_1(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<7, 7>, 64, 2, 0>,
                              MixCfg<MixSched<7, 7>, 64, 1, 0>>());  // 49
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 8>, 32, 3, 9>,
                              MixCfg<MixSched<9, 8>, 32, 2, 9>>());  // 72
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 10>, 32, 3, 0>,
                              MixCfg<MixSched<10, 10>, 32, 2, 0>>());  // 100
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 9>, 32, 2, 0>,
                              MixCfg<MixSched<15, 9>, 16, 2, 15>>());  // 135
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 7>, 32, 3, 0>,
                              MixCfg<MixSched<25, 7>, 16, 2, 0>>());  // 175
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 14>, 32, 1, 16>,
                              MixCfg<MixSched<16, 14>, 16, 2, 16>>());  // 224
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 15>, 16, 2, 18>,
                              MixCfg<MixSched<18, 15>, 8, 3, 18>>());  // 270
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 16>, 16, 2, 0>,
                              MixCfg<MixSched<21, 16>, 8, 2, 21>>());  // 336
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 20>, 16, 2, 0>,
                              MixCfg<MixSched<20, 20>, 8, 2, 0>>());  // 400
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 18>, 16, 2, 0>,
                              MixCfg<MixSched<27, 18>, 8, 1, 27>>());  // 486
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 21>, 8, 3, 27>,
                              MixCfg<MixSched<27, 21>, 4, 2, 27>>());  // 567
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 24>, 8, 3, 28>,
                              MixCfg<MixSched<28, 24>, 4, 2, 28>>());  // 672
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 27>, 8, 3, 28>,
                              MixCfg<MixSched<28, 27>, 4, 2, 28>>());  // 756
  v.push_back(mix_rows_entry<MixCfg<MixSched<42, 21>, 8, 2, 0>,
                              MixCfg<MixSched<42, 21>, 4, 2, 0>>());  // 882
  v.push_back(mix_rows_entry<MixCfg<MixSched<36, 28>, 4, 3, 36>,
                              MixCfg<MixSched<36, 28>, 2, 3, 0>>());  // 1008
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 12, 8>, 4, 2, 0>,
                              MixCfg<MixSched<12, 12, 8>, 2, 2, 0>>());  // 1152
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 12, 9>, 4, 1, 0>,
                              MixCfg<MixSched<12, 12, 9>, 2, 2, 0>>());  // 1296
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14, 7>, 4, 1, 0>,
                              MixCfg<MixSched<15, 14, 7>, 2, 1, 0>>());  // 1470
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12, 10>, 4, 1, 0>,
                              MixCfg<MixSched<14, 12, 10>, 2, 1, 0>>());  // 1680
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15, 5>, 4, 2, 0>,
                              MixCfg<MixSched<25, 15, 5>, 2, 2, 0>>());  // 1875
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 14, 7>, 2, 3, 0>,
                              MixCfg<MixSched<21, 14, 7>, 1, 2, 0>>());  // 2058
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 12, 12>, 2, 2, 0>,
                              MixCfg<MixSched<16, 12, 12>, 1, 2, 0>>());  // 2304
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 16, 10>, 2, 2, 0>,
                              MixCfg<MixSched<16, 16, 10>, 1, 2, 0>>());  // 2560
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 15, 9>, 2, 2, 0>,
                              MixCfg<MixSched<21, 15, 9>, 1, 2, 0>>());  // 2835
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 25, 5>, 2, 2, 0>,
                              MixCfg<MixSched<25, 25, 5>, 1, 3, 0>>());  // 3125
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 14, 7>, 2, 2, 0>,
                              MixCfg<MixSched<35, 14, 7>, 1, 1, 0>>());  // 3430
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15, 10>, 2, 2, 0>,
                              MixCfg<MixSched<25, 15, 10>, 1, 2, 0>>());  // 3750
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 15, 15>, 1, 2, 0>,
                              MixCfg<MixSched<18, 15, 15>, 1, 1, 0>>());  // 4050
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 15, 15>, 1, 2, 0>,
                              MixCfg<MixSched<20, 15, 15>, 1, 1, 0>>());  // 4500
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 14, 14>, 1, 3, 0>,
                              MixCfg<MixSched<25, 14, 14>, 1, 1, 0>>());  // 4900
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 18, 14>, 1, 2, 0>,
                              MixCfg<MixSched<21, 18, 14>, 1, 1, 0>>());  // 5292
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18, 18>, 1, 2, 0>,
                              MixCfg<MixSched<18, 18, 18>, 1, 1, 0>>());  // 5832
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 25, 10>, 1, 2, 0>>());  // 6250
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 18, 15>, 1, 2, 0>>());  // 6750
  v.push_back(mix_rows_entry64<MixCfg<MixSched<49, 21, 7>, 1, 2, 0>>());  // 7203
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 21, 15>, 1, 1, 0>>());  // 7875
  v.push_back(mix_rows_entry64<MixCfg<MixSched<35, 35, 7>, 1, 2, 0>>());  // 8575
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 24, 16>, 1, 1, 0>>());  // 9216
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 25, 14>, 1, 1, 0>>());  // 9800
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 21, 20>, 1, 1, 0>>());  // 10500
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 25, 18>, 1, 1, 0>>());  // 11250
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 24, 21>, 1, 1, 0>>());  // 12096
}

}  // namespace gfft
