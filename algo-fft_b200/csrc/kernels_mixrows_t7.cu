// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_7(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<8, 8>, 64, 2, 0>,
                              MixCfg<MixSched<8, 8>, 32, 3, 0>>());  // 64
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 8>, 64, 1, 0>,
                              MixCfg<MixSched<12, 8>, 32, 2, 0>>());  // 96
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 9>, 32, 2, 0>,
                              MixCfg<MixSched<14, 9>, 16, 2, 14>>());  // 126
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 9>, 32, 2, 0>,
                              MixCfg<MixSched<18, 9>, 16, 3, 0>>());  // 162
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 14>, 32, 1, 15>,
                              MixCfg<MixSched<15, 14>, 16, 2, 15>>());  // 210
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 14>, 16, 3, 0>,
                              MixCfg<MixSched<18, 14>, 8, 3, 18>>());  // 252
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 16>, 16, 2, 0>,
                              MixCfg<MixSched<20, 16>, 8, 2, 20>>());  // 320
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 16>, 16, 2, 0>,
                              MixCfg<MixSched<24, 16>, 8, 2, 0>>());  // 384
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 18>, 16, 2, 0>,
                              MixCfg<MixSched<25, 18>, 8, 1, 25>>());  // 450
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 20>, 8, 3, 0>,
                              MixCfg<MixSched<27, 20>, 4, 2, 27>>());  // 540
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 20>, 8, 3, 0>,
                              MixCfg<MixSched<32, 20>, 4, 2, 32>>());  // 640
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 21>, 8, 2, 0>,
                              MixCfg<MixSched<35, 21>, 4, 2, 0>>());  // 735
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 27>, 8, 2, 32>,
                              MixCfg<MixSched<32, 27>, 4, 2, 32>>());  // 864
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 28>, 8, 2, 35>,
                              MixCfg<MixSched<35, 28>, 4, 1, 0>>());  // 980
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 5>, 4, 2, 0>,
                              MixCfg<MixSched<15, 15, 5>, 2, 3, 0>>());  // 1125
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 10, 9>, 4, 2, 0>,
                              MixCfg<MixSched<14, 10, 9>, 2, 2, 0>>());  // 1260
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 12, 10>, 4, 1, 0>,
                              MixCfg<MixSched<12, 12, 10>, 2, 1, 0>>());  // 1440
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 10, 10>, 4, 1, 0>,
                              MixCfg<MixSched<16, 10, 10>, 2, 2, 0>>());  // 1600
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 14, 8>, 4, 1, 0>,
                              MixCfg<MixSched<16, 14, 8>, 2, 1, 0>>());  // 1792
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 12, 12>, 2, 2, 0>,
                              MixCfg<MixSched<14, 12, 12>, 1, 2, 0>>());  // 2016
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 10>, 2, 2, 0>,
                              MixCfg<MixSched<15, 15, 10>, 1, 2, 0>>());  // 2250
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 10, 10>, 2, 2, 0>,
                              MixCfg<MixSched<25, 10, 10>, 1, 2, 0>>());  // 2500
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14, 14>, 2, 2, 0>,
                              MixCfg<MixSched<14, 14, 14>, 1, 2, 0>>());  // 2744
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 16, 12>, 2, 1, 0>,
                              MixCfg<MixSched<16, 16, 12>, 1, 2, 0>>());  // 3072
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 15, 15>, 2, 1, 0>,
                              MixCfg<MixSched<15, 15, 15>, 1, 2, 0>>());  // 3375
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 15, 9>, 2, 2, 0>,
                              MixCfg<MixSched<27, 15, 9>, 1, 2, 0>>());  // 3645
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 20, 10>, 1, 3, 0>,
                              MixCfg<MixSched<20, 20, 10>, 1, 2, 0>>());  // 4000
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 15, 14>, 1, 2, 0>,
                              MixCfg<MixSched<21, 15, 14>, 1, 1, 0>>());  // 4410
  v.push_back(mix_rows_entry<MixCfg<MixSched<49, 14, 7>, 1, 3, 0>,
                              MixCfg<MixSched<49, 14, 7>, 1, 1, 0>>());  // 4802
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 18, 16>, 1, 2, 0>,
                              MixCfg<MixSched<18, 18, 16>, 1, 1, 0>>());  // 5184
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 18, 15>, 1, 2, 0>,
                              MixCfg<MixSched<21, 18, 15>, 1, 1, 0>>());  // 5670
  v.push_back(mix_rows_entry<MixCfg<MixSched<24, 16, 16>, 1, 2, 0>,
                              MixCfg<MixSched<24, 16, 16>, 1, 1, 0>>());  // 6144
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 21, 15>, 1, 2, 0>>());  // 6615
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 16, 16>, 1, 2, 0>>());  // 7168
  v.push_back(mix_rows_entry64<MixCfg<MixSched<24, 18, 18>, 1, 1, 0>>());  // 7776
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 20, 20>, 1, 1, 0>>());  // 8400
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 20, 18>, 1, 1, 0>>());  // 9000
  v.push_back(mix_rows_entry64<MixCfg<MixSched<49, 14, 14>, 1, 1, 0>>());  // 9604
  v.push_back(mix_rows_entry64<MixCfg<MixSched<35, 21, 14>, 1, 1, 0>>());  // 10290
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 21, 21>, 1, 1, 0>>());  // 11025
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 24, 20>, 1, 1, 0>>());  // 12000
}

}  // namespace gfft
