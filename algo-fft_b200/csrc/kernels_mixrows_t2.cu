// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_2(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 5>, 64, 3, 0>,
                              MixCfg<MixSched<10, 5>, 64, 2, 0>>());  // 50
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 5>, 64, 2, 0>,
                              MixCfg<MixSched<15, 5>, 32, 3, 0>>());  // 75
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 7>, 64, 1, 0>,
                              MixCfg<MixSched<15, 7>, 32, 1, 0>>());  // 105
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 10>, 32, 2, 0>,
                              MixCfg<MixSched<14, 10>, 16, 2, 14>>());  // 140
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 12>, 32, 1, 15>,
                              MixCfg<MixSched<15, 12>, 16, 2, 15>>());  // 180
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15>, 32, 1, 0>,
                              MixCfg<MixSched<15, 15>, 16, 2, 0>>());  // 225
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 14>, 16, 3, 0>,
                              MixCfg<MixSched<20, 14>, 8, 2, 20>>());  // 280
  v.push_back(mix_rows_entry<MixCfg<MixSched<49, 7>, 16, 3, 0>,
                              MixCfg<MixSched<49, 7>, 8, 3, 0>>());  // 343
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 15>, 16, 2, 0>,
                              MixCfg<MixSched<27, 15>, 8, 2, 0>>());  // 405
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 14>, 16, 2, 0>,
                              MixCfg<MixSched<35, 14>, 8, 1, 0>>());  // 490
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 24>, 8, 3, 0>,
                              MixCfg<MixSched<24, 24>, 4, 4, 0>>());  // 576
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 25>, 8, 3, 27>,
                              MixCfg<MixSched<27, 25>, 4, 2, 27>>());  // 675
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 24>, 8, 2, 0>,
                              MixCfg<MixSched<32, 24>, 4, 2, 32>>());  // 768
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 28>, 8, 2, 32>,
                              MixCfg<MixSched<32, 28>, 4, 2, 32>>());  // 896
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 32>, 4, 4, 0>,
                              MixCfg<MixSched<32, 32>, 2, 4, 0>>());  // 1024
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12, 7>, 4, 2, 0>,
                              MixCfg<MixSched<14, 12, 7>, 2, 2, 0>>());  // 1176
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 9, 7>, 4, 2, 0>,
                              MixCfg<MixSched<21, 9, 7>, 2, 2, 0>>());  // 1323
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 10, 10>, 4, 1, 0>,
                              MixCfg<MixSched<15, 10, 10>, 2, 2, 0>>());  // 1500
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 9, 9>, 4, 1, 0>,
                              MixCfg<MixSched<21, 9, 9>, 2, 1, 0>>());  // 1701
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14, 9>, 4, 1, 0>,
                              MixCfg<MixSched<15, 14, 9>, 2, 1, 0>>());  // 1890
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14, 10>, 2, 2, 0>,
                              MixCfg<MixSched<15, 14, 10>, 1, 2, 0>>());  // 2100
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14, 12>, 2, 2, 0>,
                              MixCfg<MixSched<14, 14, 12>, 1, 2, 0>>());  // 2352
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 12, 12>, 2, 2, 0>,
                              MixCfg<MixSched<18, 12, 12>, 1, 2, 0>>());  // 2592
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 15, 12>, 2, 1, 0>,
                              MixCfg<MixSched<16, 15, 12>, 1, 1, 0>>());  // 2880
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 14, 14>, 2, 1, 0>,
                              MixCfg<MixSched<16, 14, 14>, 1, 1, 0>>());  // 3136
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 16, 12>, 2, 1, 0>,
                              MixCfg<MixSched<18, 16, 12>, 1, 1, 0>>());  // 3456
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 15, 14>, 2, 1, 0>,
                              MixCfg<MixSched<18, 15, 14>, 1, 1, 0>>());  // 3780
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 14, 14>, 1, 3, 0>,
                              MixCfg<MixSched<21, 14, 14>, 1, 1, 0>>());  // 4116
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18, 14>, 1, 2, 0>,
                              MixCfg<MixSched<18, 18, 14>, 1, 1, 0>>());  // 4536
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 20, 10>, 1, 2, 0>,
                              MixCfg<MixSched<25, 20, 10>, 1, 1, 0>>());  // 5000
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 16, 16>, 1, 2, 0>,
                              MixCfg<MixSched<21, 16, 16>, 1, 1, 0>>());  // 5376
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 20, 14>, 1, 1, 0>,
                              MixCfg<MixSched<21, 20, 14>, 1, 1, 0>>());  // 5880
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 16, 14>, 1, 2, 0>>());  // 6272
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 18, 18>, 1, 1, 0>>());  // 6804
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 18, 15>, 1, 2, 0>>());  // 7290
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 21, 18>, 1, 1, 0>>());  // 7938
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 20, 18>, 1, 1, 0>>());  // 8640
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 21, 21>, 1, 1, 0>>());  // 9261
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 20, 20>, 1, 1, 0>>());  // 10000
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 21, 21>, 1, 1, 0>>());  // 10584
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 21, 20>, 1, 1, 0>>());  // 11340
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 25, 18>, 1, 1, 0>>());  // 12150
}

}  // namespace gfft
