// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_1(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<7, 7>, 64, 2, 0>,
                              MixCfg<MixSched<7, 7>, 64, 1, 0>>());  // 49
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 6>, 64, 2, 0>,
                              MixCfg<MixSched<10, 6>, 32, 3, 0>>());  // 60
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 8>, 32, 3, 9>,
                              MixCfg<MixSched<9, 8>, 32, 2, 9>>());  // 72
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 7>, 64, 2, 0>,
                              MixCfg<MixSched<12, 7>, 32, 2, 0>>());  // 84
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 10>, 32, 3, 0>,
                              MixCfg<MixSched<10, 10>, 32, 2, 0>>());  // 100
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 10>, 32, 2, 12>,
                              MixCfg<MixSched<12, 10>, 16, 3, 12>>());  // 120
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 9>, 32, 2, 0>,
                              MixCfg<MixSched<15, 9>, 16, 2, 15>>());  // 135
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 10>, 32, 2, 0>,
                              MixCfg<MixSched<15, 10>, 16, 2, 15>>());  // 150
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 7>, 32, 3, 0>,
                              MixCfg<MixSched<25, 7>, 16, 2, 0>>());  // 175
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14>, 32, 2, 0>,
                              MixCfg<MixSched<14, 14>, 16, 2, 0>>());  // 196
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 14>, 32, 1, 16>,
                              MixCfg<MixSched<16, 14>, 16, 2, 16>>());  // 224
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 7>, 32, 2, 0>,
                              MixCfg<MixSched<35, 7>, 16, 2, 0>>());  // 245
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 15>, 16, 2, 18>,
                              MixCfg<MixSched<18, 15>, 8, 3, 18>>());  // 270
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 15>, 16, 2, 0>,
                              MixCfg<MixSched<20, 15>, 8, 2, 20>>());  // 300
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 16>, 16, 2, 0>,
                              MixCfg<MixSched<21, 16>, 8, 2, 21>>());  // 336
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15>, 16, 2, 0>,
                              MixCfg<MixSched<25, 15>, 8, 2, 0>>());  // 375
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 20>, 16, 2, 0>,
                              MixCfg<MixSched<20, 20>, 8, 2, 0>>());  // 400
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 21>, 16, 2, 0>,
                              MixCfg<MixSched<21, 21>, 8, 2, 0>>());  // 441
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 18>, 16, 2, 0>,
                              MixCfg<MixSched<27, 18>, 8, 1, 27>>());  // 486
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 16>, 8, 4, 0>,
                              MixCfg<MixSched<32, 16>, 4, 4, 0>>());  // 512
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 21>, 8, 3, 27>,
                              MixCfg<MixSched<27, 21>, 4, 2, 27>>());  // 567
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 25>, 8, 3, 0>,
                              MixCfg<MixSched<25, 25>, 4, 3, 0>>());  // 625
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 24>, 8, 3, 28>,
                              MixCfg<MixSched<28, 24>, 4, 2, 28>>());  // 672
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 24>, 8, 2, 30>,
                              MixCfg<MixSched<30, 24>, 4, 2, 30>>());  // 720
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 27>, 8, 3, 28>,
                              MixCfg<MixSched<28, 27>, 4, 2, 28>>());  // 756
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 27>, 8, 2, 30>,
                              MixCfg<MixSched<30, 27>, 4, 2, 30>>());  // 810
  v.push_back(mix_rows_entry<MixCfg<MixSched<42, 21>, 8, 2, 0>,
                              MixCfg<MixSched<42, 21>, 4, 2, 0>>());  // 882
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 30>, 8, 2, 32>,
                              MixCfg<MixSched<32, 30>, 4, 2, 32>>());  // 960
  v.push_back(mix_rows_entry<MixCfg<MixSched<36, 28>, 4, 3, 36>,
                              MixCfg<MixSched<36, 28>, 2, 3, 0>>());  // 1008
}

}  // namespace gfft
