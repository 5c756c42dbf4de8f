// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_part_6(std::vector<MixEntry>& v) {
  v.push_back(mix_entry<MixCfg<MixSched<9, 7>, 16, 7, 0>,
                         MixCfg<MixSched<9, 7>, 16, 7, 0>,
                         MixCfg<MixSched<9, 7>, 8, 7, 9>,
                         MixCfg<MixSched<9, 7>, 8, 7, 9>>());  // 63
  v.push_back(mix_entry<MixCfg<MixSched<10, 9>, 16, 6, 10>,
                         MixCfg<MixSched<10, 9>, 16, 6, 10>,
                         MixCfg<MixSched<10, 9>, 8, 7, 10>,
                         MixCfg<MixSched<10, 9>, 8, 7, 10>>());  // 90
  v.push_back(mix_entry<MixCfg<MixSched<25, 5>, 16, 7, 0>,
                         MixCfg<MixSched<25, 5>, 16, 7, 0>,
                         MixCfg<MixSched<25, 5>, 8, 6, 0>,
                         MixCfg<MixSched<25, 5>, 8, 6, 0>>());  // 125
  v.push_back(mix_entry<MixCfg<MixSched<16, 10>, 16, 5, 0>,
                         MixCfg<MixSched<16, 10>, 16, 5, 0>,
                         MixCfg<MixSched<16, 10>, 8, 4, 16>,
                         MixCfg<MixSched<16, 10>, 8, 4, 16>>());  // 160
  v.push_back(mix_entry<MixCfg<MixSched<20, 10>, 16, 5, 0>,
                         MixCfg<MixSched<20, 10>, 16, 5, 0>,
                         MixCfg<MixSched<20, 10>, 8, 4, 0>,
                         MixCfg<MixSched<20, 10>, 8, 4, 0>>());  // 200
  v.push_back(mix_entry<MixCfg<MixSched<25, 10>, 16, 4, 0>,
                         MixCfg<MixSched<25, 10>, 16, 4, 0>,
                         MixCfg<MixSched<25, 10>, 8, 3, 0>,
                         MixCfg<MixSched<25, 10>, 8, 3, 0>>());  // 250
  v.push_back(mix_entry<MixCfg<MixSched<21, 15>, 16, 2, 0>,
                         MixCfg<MixSched<21, 15>, 16, 2, 0>,
                         MixCfg<MixSched<21, 15>, 8, 2, 21>,
                         MixCfg<MixSched<21, 15>, 8, 2, 21>>());  // 315
  v.push_back(mix_entry<MixCfg<MixSched<21, 18>, 16, 2, 21>,
                         MixCfg<MixSched<21, 18>, 16, 2, 21>,
                         MixCfg<MixSched<21, 18>, 8, 2, 21>,
                         MixCfg<MixSched<21, 18>, 8, 2, 21>>());  // 378
  v.push_back(mix_entry<MixCfg<MixSched<28, 16>, 16, 2, 0>,
                         MixCfg<MixSched<28, 16>, 16, 2, 0>,
                         MixCfg<MixSched<28, 16>, 8, 2, 0>,
                         MixCfg<MixSched<28, 16>, 8, 2, 0>>());  // 448
  v.push_back(mix_entry<MixCfg<MixSched<25, 21>, 8, 3, 25>,
                         MixCfg<MixSched<25, 21>, 8, 3, 25>,
                         MixCfg<MixSched<25, 21>, 4, 3, 25>,
                         MixCfg<MixSched<25, 21>, 4, 3, 25>>());  // 525
  v.push_back(mix_entry<MixCfg<MixSched<30, 21>, 8, 2, 30>,
                         MixCfg<MixSched<30, 21>, 8, 2, 30>,
                         MixCfg<MixSched<30, 21>, 4, 2, 30>,
                         MixCfg<MixSched<30, 21>, 4, 2, 30>>());  // 630
  v.push_back(mix_entry<MixCfg<MixSched<27, 27>, 8, 3, 0>,
                         MixCfg<MixSched<27, 27>, 8, 3, 0>,
                         MixCfg<MixSched<27, 27>, 4, 2, 0>,
                         MixCfg<MixSched<27, 27>, 4, 2, 0>>());  // 729
  v.push_back(mix_entry<MixCfg<MixSched<30, 28>, 8, 2, 30>,
                         MixCfg<MixSched<30, 28>, 8, 2, 30>,
                         MixCfg<MixSched<30, 28>, 4, 2, 30>,
                         MixCfg<MixSched<30, 28>, 4, 2, 30>>());  // 840
  v.push_back(mix_entry<MixCfg<MixSched<36, 27>, 8, 2, 36>,
                         MixCfg<MixSched<36, 27>, 8, 2, 36>,
                         MixCfg<MixSched<36, 27>, 4, 1, 0>,
                         MixCfg<MixSched<36, 27>, 4, 1, 0>>());  // 972
}

}  // namespace gfft
