// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_5(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<10, 6>, 16, 8, 0>,
                         MixCfg<MixSched<10, 6>, 16, 8, 0>,
                         MixCfg<MixSched<10, 6>, 8, 8, 0>,
                         MixCfg<MixSched<10, 6>, 8, 8, 0>>());  // 60
  v.push_back(mix_entry<MixCfg<MixSched<12, 7>, 16, 7, 0>,
                         MixCfg<MixSched<12, 7>, 16, 7, 0>,
                         MixCfg<MixSched<12, 7>, 8, 8, 0>,
                         MixCfg<MixSched<12, 7>, 8, 8, 0>>());  // 84
  v.push_back(mix_entry<MixCfg<MixSched<12, 10>, 16, 5, 12>,
                         MixCfg<MixSched<12, 10>, 16, 5, 12>,
                         MixCfg<MixSched<12, 10>, 8, 6, 12>,
                         MixCfg<MixSched<12, 10>, 8, 6, 12>>());  // 120
  v.push_back(mix_entry<MixCfg<MixSched<15, 10>, 16, 5, 0>,
                         MixCfg<MixSched<15, 10>, 16, 5, 0>,
                         MixCfg<MixSched<15, 10>, 8, 4, 15>,
                         MixCfg<MixSched<15, 10>, 8, 4, 15>>());  // 150
  v.push_back(mix_entry<MixCfg<MixSched<14, 14>, 16, 4, 0>,
                         MixCfg<MixSched<14, 14>, 16, 4, 0>,
                         MixCfg<MixSched<14, 14>, 8, 4, 0>,
                         MixCfg<MixSched<14, 14>, 8, 4, 0>>());  // 196
  v.push_back(mix_entry<MixCfg<MixSched<35, 7>, 16, 4, 0>,
                         MixCfg<MixSched<35, 7>, 16, 4, 0>,
                         MixCfg<MixSched<35, 7>, 8, 4, 0>,
                         MixCfg<MixSched<35, 7>, 8, 4, 0>>());  // 245
  v.push_back(mix_entry<MixCfg<MixSched<20, 15>, 16, 2, 0>,
                         MixCfg<MixSched<20, 15>, 16, 2, 0>,
                         MixCfg<MixSched<20, 15>, 8, 2, 20>,
                         MixCfg<MixSched<20, 15>, 8, 2, 20>>());  // 300
  v.push_back(mix_entry<MixCfg<MixSched<25, 15>, 16, 2, 0>,
                         MixCfg<MixSched<25, 15>, 16, 2, 0>,
                         MixCfg<MixSched<25, 15>, 8, 2, 0>,
                         MixCfg<MixSched<25, 15>, 8, 2, 0>>());  // 375
  v.push_back(mix_entry<MixCfg<MixSched<21, 21>, 16, 2, 0>,
                         MixCfg<MixSched<21, 21>, 16, 2, 0>,
                         MixCfg<MixSched<21, 21>, 8, 2, 0>,
                         MixCfg<MixSched<21, 21>, 8, 2, 0>>());  // 441
  v.push_back(mix_entry<MixCfg<MixSched<32, 16>, 8, 4, 0>,
                         MixCfg<MixSched<32, 16>, 8, 4, 0>,
                         MixCfg<MixSched<32, 16>, 4, 4, 0>,
                         MixCfg<MixSched<8, 8, 8>, 8, 2, 0>>());  // 512
  v.push_back(mix_entry<MixCfg<MixSched<25, 25>, 8, 3, 0>,
                         MixCfg<MixSched<25, 25>, 8, 3, 0>,
                         MixCfg<MixSched<25, 25>, 4, 3, 0>,
                         MixCfg<MixSched<25, 25>, 4, 3, 0>>());  // 625
  v.push_back(mix_entry<MixCfg<MixSched<30, 24>, 8, 2, 30>,
                         MixCfg<MixSched<30, 24>, 8, 2, 30>,
                         MixCfg<MixSched<30, 24>, 4, 2, 30>,
                         MixCfg<MixSched<30, 24>, 4, 2, 30>>());  // 720
  v.push_back(mix_entry<MixCfg<MixSched<30, 27>, 8, 2, 30>,
                         MixCfg<MixSched<30, 27>, 8, 2, 30>,
                         MixCfg<MixSched<30, 27>, 4, 2, 30>,
                         MixCfg<MixSched<30, 27>, 4, 2, 30>>());  // 810
  v.push_back(mix_entry<MixCfg<MixSched<32, 30>, 8, 2, 32>,
                         MixCfg<MixSched<32, 30>, 8, 2, 32>,
                         MixCfg<MixSched<32, 30>, 4, 2, 32>,
                         MixCfg<MixSched<32, 30>, 4, 2, 32>>());  // 960
}

}  // namespace gfft
