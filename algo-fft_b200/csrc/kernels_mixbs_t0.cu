// Generated by gen_mixcols.py; do not edit.
#include "kernels_mixcols.cuh"

namespace gfft {

void mix_bs_part_0(std::vector<MixBsEntry>& v) {
  v.push_back(mix_bs_entry<MixCfg<MixSched<10, 8>, 16, 7, 0>,
                            MixCfg<MixSched<10, 8>, 8, 7, 10>>());  // 80
  v.push_back(mix_bs_entry<MixCfg<MixSched<12, 12>, 16, 5, 0>,
                            MixCfg<MixSched<12, 12>, 8, 6, 0>>());  // 144
  v.push_back(mix_bs_entry<MixCfg<MixSched<16, 14>, 16, 3, 16>,
                            MixCfg<MixSched<16, 14>, 8, 4, 16>>());  // 224
  v.push_back(mix_bs_entry<MixCfg<MixSched<18, 16>, 16, 2, 18>,
                            MixCfg<MixSched<18, 16>, 8, 3, 18>>());  // 288
  v.push_back(mix_bs_entry<MixCfg<MixSched<24, 16>, 16, 2, 0>,
                            MixCfg<MixSched<24, 16>, 8, 2, 0>>());  // 384
  v.push_back(mix_bs_entry<MixCfg<MixSched<28, 16>, 16, 2, 0>,
                            MixCfg<MixSched<28, 16>, 8, 2, 0>>());  // 448
}

}  // namespace gfft
