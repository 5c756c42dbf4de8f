// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_4(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<8, 7>, 64, 2, 8>,
                              MixCfg<MixSched<8, 7>, 64, 1, 8>>());  // 56
  v.push_back(mix_rows_entry<MixCfg<MixSched<9, 9>, 32, 3, 0>,
                              MixCfg<MixSched<9, 9>, 32, 2, 0>>());  // 81
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 8>, 64, 1, 0>,
                              MixCfg<MixSched<14, 8>, 32, 2, 0>>());  // 112
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 7>, 32, 3, 0>,
                              MixCfg<MixSched<21, 7>, 16, 3, 0>>());  // 147
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 12>, 32, 1, 16>,
                              MixCfg<MixSched<16, 12>, 16, 2, 0>>());  // 192
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 9>, 32, 2, 0>,
                              MixCfg<MixSched<27, 9>, 16, 2, 0>>());  // 243
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 14>, 16, 3, 0>,
                              MixCfg<MixSched<21, 14>, 8, 2, 0>>());  // 294
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 18>, 16, 2, 20>,
                              MixCfg<MixSched<20, 18>, 8, 2, 20>>());  // 360
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 18>, 16, 2, 0>,
                              MixCfg<MixSched<24, 18>, 8, 2, 24>>());  // 432
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 21>, 8, 3, 24>,
                              MixCfg<MixSched<24, 21>, 4, 4, 24>>());  // 504
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 24>, 8, 3, 25>,
                              MixCfg<MixSched<25, 24>, 4, 3, 25>>());  // 600
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 25>, 8, 3, 28>,
                              MixCfg<MixSched<28, 25>, 4, 2, 28>>());  // 700
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 25>, 8, 2, 32>,
                              MixCfg<MixSched<32, 25>, 4, 2, 32>>());  // 800
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 27>, 8, 2, 35>,
                              MixCfg<MixSched<35, 27>, 4, 1, 0>>());  // 945
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 10, 7>, 4, 2, 0>,
                              MixCfg<MixSched<15, 10, 7>, 2, 2, 0>>());  // 1050
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 9, 9>, 4, 2, 0>,
                              MixCfg<MixSched<15, 9, 9>, 2, 2, 0>>());  // 1215
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 10, 9>, 4, 2, 0>,
                              MixCfg<MixSched<15, 10, 9>, 2, 2, 0>>());  // 1350
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 12, 8>, 4, 1, 0>,
                              MixCfg<MixSched<16, 12, 8>, 2, 2, 0>>());  // 1536
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 12, 12>, 2, 3, 0>,
                              MixCfg<MixSched<12, 12, 12>, 2, 2, 0>>());  // 1728
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 12, 9>, 2, 3, 0>,
                              MixCfg<MixSched<18, 12, 9>, 1, 3, 0>>());  // 1944
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 9, 9>, 2, 3, 0>,
                              MixCfg<MixSched<27, 9, 9>, 1, 3, 0>>());  // 2187
  v.push_back(mix_rows_entry<MixCfg<MixSched<49, 7, 7>, 2, 3, 0>,
                              MixCfg<MixSched<49, 7, 7>, 1, 3, 0>>());  // 2401
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 14, 9>, 2, 2, 0>,
                              MixCfg<MixSched<21, 14, 9>, 1, 2, 0>>());  // 2646
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14, 14>, 2, 1, 0>,
                              MixCfg<MixSched<15, 14, 14>, 1, 1, 0>>());  // 2940
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 16, 10>, 2, 1, 0>,
                              MixCfg<MixSched<20, 16, 10>, 1, 1, 0>>());  // 3200
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 14, 14>, 2, 1, 0>,
                              MixCfg<MixSched<18, 14, 14>, 1, 1, 0>>());  // 3528
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18, 12>, 1, 3, 0>,
                              MixCfg<MixSched<18, 18, 12>, 1, 1, 0>>());  // 3888
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 16, 15>, 1, 2, 0>,
                              MixCfg<MixSched<18, 16, 15>, 1, 1, 0>>());  // 4320
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 16, 14>, 1, 2, 0>,
                              MixCfg<MixSched<21, 16, 14>, 1, 1, 0>>());  // 4704
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 21, 9>, 1, 2, 0>,
                              MixCfg<MixSched<27, 21, 9>, 1, 1, 0>>());  // 5103
  v.push_back(mix_rows_entry<MixCfg<MixSched<28, 14, 14>, 1, 3, 0>,
                              MixCfg<MixSched<28, 14, 14>, 1, 1, 0>>());  // 5488
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 18, 16>, 1, 2, 0>,
                              MixCfg<MixSched<21, 18, 16>, 1, 1, 0>>());  // 6048
  v.push_back(mix_rows_entry64<MixCfg<MixSched<20, 20, 16>, 1, 1, 0>>());  // 6400
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 18, 16>, 1, 2, 0>>());  // 6912
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 20, 15>, 1, 1, 0>>());  // 7500
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 21, 16>, 1, 1, 0>>());  // 8064
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 25, 14>, 1, 1, 0>>());  // 8750
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 21, 16>, 1, 1, 0>>());  // 9408
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 25, 15>, 1, 1, 0>>());  // 10125
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 24, 18>, 1, 1, 0>>());  // 10800
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 24, 18>, 1, 1, 0>>());  // 11664
  v.push_back(mix_rows_entry64<MixCfg<MixSched<32, 24, 16>, 1, 1, 0>>());  // 12288
}

}  // namespace gfft
