// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_bs_part_2(std::vector<MixBsEntry>& v) {
  v.push_back(mix_bs_entry<MixCfg<MixSched<16, 8>, 16, 7, 0>,
                            MixCfg<MixSched<16, 8>, 8, 8, 0>>());  // 128
  v.push_back(mix_bs_entry<MixCfg<MixSched<16, 12>, 16, 3, 16>,
                            MixCfg<MixSched<16, 12>, 8, 4, 0>>());  // 192
  v.push_back(mix_bs_entry<MixCfg<MixSched<16, 16>, 16, 3, 0>,
                            MixCfg<MixSched<16, 16>, 8, 4, 0>>());  // 256
  v.push_back(mix_bs_entry<MixCfg<MixSched<21, 16>, 16, 2, 0>,
                            MixCfg<MixSched<21, 16>, 8, 2, 21>>());  // 336
  v.push_back(mix_bs_entry<MixCfg<MixSched<24, 18>, 16, 2, 0>,
                            MixCfg<MixSched<24, 18>, 8, 2, 24>>());  // 432
  v.push_back(mix_bs_entry<MixCfg<MixSched<32, 16>, 8, 4, 0>,
                            MixCfg<MixSched<32, 16>, 4, 4, 0>>());  // 512
}

}  // namespace gfft
