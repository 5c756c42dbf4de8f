// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_6(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 7>, 64, 2, 0>,
                              MixCfg<MixSched<9, 7>, 32, 2, 9>>());  // 63
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 9>, 32, 3, 10>,
                              MixCfg<MixSched<10, 9>, 32, 2, 10>>());  // 90
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 5>, 64, 2, 0>,
                              MixCfg<MixSched<25, 5>, 32, 2, 0>>());  // 125
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 10>, 32, 2, 0>,
                              MixCfg<MixSched<16, 10>, 16, 2, 16>>());  // 160
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 10>, 32, 2, 0>,
                              MixCfg<MixSched<20, 10>, 16, 2, 0>>());  // 200
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 10>, 32, 2, 0>,
                              MixCfg<MixSched<25, 10>, 16, 2, 0>>());  // 250
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 15>, 16, 2, 0>,
                              MixCfg<MixSched<21, 15>, 8, 2, 21>>());  // 315
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 18>, 16, 2, 21>,
                              MixCfg<MixSched<21, 18>, 8, 2, 21>>());  // 378
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 16>, 16, 2, 0>,
                              MixCfg<MixSched<28, 16>, 8, 2, 0>>());  // 448
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 21>, 8, 3, 25>,
                              MixCfg<MixSched<25, 21>, 4, 3, 25>>());  // 525
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 21>, 8, 2, 30>,
                              MixCfg<MixSched<30, 21>, 4, 2, 30>>());  // 630
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 27>, 8, 3, 0>,
                              MixCfg<MixSched<27, 27>, 4, 2, 0>>());  // 729
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 28>, 8, 2, 30>,
                              MixCfg<MixSched<30, 28>, 4, 2, 30>>());  // 840
  v.push_back(mix_rows_entry<MixCfg<MixSched<36, 27>, 8, 2, 36>,
                              MixCfg<MixSched<36, 27>, 4, 1, 0>>());  // 972
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 10, 8>, 4, 2, 0>,
                              MixCfg<MixSched<14, 10, 8>, 2, 2, 0>>());  // 1120
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 10, 5>, 4, 2, 0>,
                              MixCfg<MixSched<25, 10, 5>, 2, 2, 0>>());  // 1250
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 10, 10>, 4, 1, 0>,
                              MixCfg<MixSched<14, 10, 10>, 2, 2, 0>>());  // 1400
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 7>, 4, 1, 0>,
                              MixCfg<MixSched<15, 15, 7>, 2, 1, 0>>());  // 1575
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14, 9>, 4, 1, 0>,
                              MixCfg<MixSched<14, 14, 9>, 2, 1, 0>>());  // 1764
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 10, 10>, 2, 3, 0>,
                              MixCfg<MixSched<20, 10, 10>, 1, 3, 0>>());  // 2000
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 14, 10>, 2, 2, 0>,
                              MixCfg<MixSched<16, 14, 10>, 1, 2, 0>>());  // 2240
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 14, 7>, 2, 3, 0>,
                              MixCfg<MixSched<25, 14, 7>, 1, 2, 0>>());  // 2450
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 12>, 2, 1, 0>,
                              MixCfg<MixSched<15, 15, 12>, 1, 2, 0>>());  // 2700
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 14, 12>, 2, 1, 0>,
                              MixCfg<MixSched<18, 14, 12>, 1, 1, 0>>());  // 3024
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 15, 14>, 2, 1, 0>,
                              MixCfg<MixSched<16, 15, 14>, 1, 1, 0>>());  // 3360
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 15, 15>, 2, 1, 0>,
                              MixCfg<MixSched<16, 15, 15>, 1, 1, 0>>());  // 3600
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 21, 9>, 2, 1, 0>,
                              MixCfg<MixSched<21, 21, 9>, 1, 1, 0>>());  // 3969
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 25, 7>, 1, 3, 0>,
                              MixCfg<MixSched<25, 25, 7>, 1, 1, 0>>());  // 4375
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 16, 15>, 1, 2, 0>,
                              MixCfg<MixSched<20, 16, 15>, 1, 1, 0>>());  // 4800
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 21, 7>, 1, 3, 0>,
                              MixCfg<MixSched<35, 21, 7>, 1, 1, 0>>());  // 5145
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15, 15>, 1, 2, 0>,
                              MixCfg<MixSched<25, 15, 15>, 1, 1, 0>>());  // 5625
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 25, 7>, 1, 2, 0>,
                              MixCfg<MixSched<35, 25, 7>, 1, 1, 0>>());  // 6125
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 27, 9>, 1, 2, 0>>());  // 6561
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 21, 16>, 1, 1, 0>>());  // 7056
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 20, 16>, 1, 1, 0>>());  // 7680
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 21, 14>, 1, 1, 0>>());  // 8232
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 20, 16>, 1, 1, 0>>());  // 8960
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 20, 20>, 1, 1, 0>>());  // 9600
  v.push_back(mix_rows_entry64<MixCfg<MixSched<32, 20, 16>, 1, 1, 0>>());  // 10240
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 28, 14>, 1, 1, 0>>());  // 10976
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 21, 21>, 1, 1, 0>>());  // 11907
}

}  // namespace gfft
