// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_rows_part_5(std::vector<MixRowsEntry>& v) {
  v.push_back(mix_rows_entry<MixCfg<MixSched<10, 6>, 64, 2, 0>,
                              MixCfg<MixSched<10, 6>, 32, 3, 0>>());  // 60
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 7>, 64, 2, 0>,
                              MixCfg<MixSched<12, 7>, 32, 2, 0>>());  // 84
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 10>, 32, 2, 12>,
                              MixCfg<MixSched<12, 10>, 16, 3, 12>>());  // 120
  v.push_back(mix_rows_entry<MixCfg<MixSched<15, 10>, 32, 2, 0>,
                              MixCfg<MixSched<15, 10>, 16, 2, 15>>());  // 150
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14>, 32, 2, 0>,
                              MixCfg<MixSched<14, 14>, 16, 2, 0>>());  // 196
  v.push_back(mix_rows_entry<MixCfg<MixSched<35, 7>, 32, 2, 0>,
                              MixCfg<MixSched<35, 7>, 16, 2, 0>>());  // 245
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 15>, 16, 2, 0>,
                              MixCfg<MixSched<20, 15>, 8, 2, 20>>());  // 300
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 15>, 16, 2, 0>,
                              MixCfg<MixSched<25, 15>, 8, 2, 0>>());  // 375
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 21>, 16, 2, 0>,
                              MixCfg<MixSched<21, 21>, 8, 2, 0>>());  // 441
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 16>, 8, 4, 0>,
                              MixCfg<MixSched<32, 16>, 4, 4, 0>>());  // 512
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 25>, 8, 3, 0>,
                              MixCfg<MixSched<25, 25>, 4, 3, 0>>());  // 625
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 24>, 8, 2, 30>,
                              MixCfg<MixSched<30, 24>, 4, 2, 30>>());  // 720
  v.push_back(mix_rows_entry<MixCfg<MixSched<30, 27>, 8, 2, 30>,
                              MixCfg<MixSched<30, 27>, 4, 2, 30>>());  // 810
  v.push_back(mix_rows_entry<MixCfg<MixSched<32, 30>, 8, 2, 32>,
                              MixCfg<MixSched<32, 30>, 4, 2, 32>>());  // 960
  v.push_back(mix_rows_entry<MixCfg<MixSched<12, 10, 9>, 4, 2, 0>,
                              MixCfg<MixSched<12, 10, 9>, 2, 2, 0>>());  // 1080
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 7, 7>, 4, 3, 0>,
                              MixCfg<MixSched<25, 7, 7>, 2, 2, 0>>());  // 1225
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14, 7>, 4, 2, 0>,
                              MixCfg<MixSched<14, 14, 7>, 2, 2, 0>>());  // 1372
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14, 8>, 4, 2, 0>,
                              MixCfg<MixSched<14, 14, 8>, 2, 2, 0>>());  // 1568
  v.push_back(mix_rows_entry<MixCfg<MixSched<25, 10, 7>, 4, 2, 0>,
                              MixCfg<MixSched<25, 10, 7>, 2, 2, 0>>());  // 1750
  v.push_back(mix_rows_entry<MixCfg<MixSched<14, 14, 10>, 2, 2, 0>,
                              MixCfg<MixSched<14, 14, 10>, 1, 2, 0>>());  // 1960
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 15, 7>, 2, 2, 0>,
                              MixCfg<MixSched<21, 15, 7>, 1, 2, 0>>());  // 2205
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 15, 9>, 2, 2, 0>,
                              MixCfg<MixSched<18, 15, 9>, 1, 2, 0>>());  // 2430
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 14, 12>, 2, 1, 0>,
                              MixCfg<MixSched<16, 14, 12>, 1, 1, 0>>());  // 2688
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 15, 10>, 2, 2, 0>,
                              MixCfg<MixSched<20, 15, 10>, 1, 2, 0>>());  // 3000
  v.push_back(mix_rows_entry<MixCfg<MixSched<18, 15, 12>, 2, 1, 0>,
                              MixCfg<MixSched<18, 15, 12>, 1, 1, 0>>());  // 3240
  v.push_back(mix_rows_entry<MixCfg<MixSched<16, 16, 14>, 2, 1, 0>,
                              MixCfg<MixSched<16, 16, 14>, 1, 1, 0>>());  // 3584
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 14, 14>, 1, 3, 0>,
                              MixCfg<MixSched<20, 14, 14>, 1, 1, 0>>());  // 3920
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 18, 9>, 1, 3, 0>,
                              MixCfg<MixSched<27, 18, 9>, 1, 1, 0>>());  // 4374
  v.push_back(mix_rows_entry<MixCfg<MixSched<21, 15, 15>, 1, 2, 0>,
                              MixCfg<MixSched<21, 15, 15>, 1, 1, 0>>());  // 4725
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 16, 16>, 1, 2, 0>,
                              MixCfg<MixSched<20, 16, 16>, 1, 1, 0>>());  // 5120
  v.push_back(mix_rows_entry<MixCfg<MixSched<20, 20, 14>, 1, 2, 0>,
                              MixCfg<MixSched<20, 20, 14>, 1, 1, 0>>());  // 5600
  v.push_back(mix_rows_entry<MixCfg<MixSched<27, 15, 15>, 1, 2, 0>,
                              MixCfg<MixSched<27, 15, 15>, 1, 1, 0>>());  // 6075
  v.push_back(mix_rows_entry64<MixCfg<MixSched<20, 18, 18>, 1, 1, 0>>());  // 6480
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 20, 14>, 1, 1, 0>>());  // 7000
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 20, 18>, 1, 1, 0>>());  // 7560
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 18, 18>, 1, 1, 0>>());  // 8100
  v.push_back(mix_rows_entry64<MixCfg<MixSched<21, 21, 20>, 1, 1, 0>>());  // 8820
  v.push_back(mix_rows_entry64<MixCfg<MixSched<25, 21, 18>, 1, 1, 0>>());  // 9450
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 21, 18>, 1, 1, 0>>());  // 10206
  v.push_back(mix_rows_entry64<MixCfg<MixSched<27, 27, 15>, 1, 1, 0>>());  // 10935
  v.push_back(mix_rows_entry64<MixCfg<MixSched<28, 21, 20>, 1, 1, 0>>());  // 11760
}

}  // namespace gfft
