// Learned-proposal form (EXEC_CHOICE 7): network shape shared by the CUDA kernels and the host.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace pct {
namespace learned {

// A small 3D CNN over two co-located 9x9x9 patches (input MRI, atlas MRI):
//   conv1 2->16, conv2..conv4 16->16, all 3x3x3 "valid" + bias + ReLU  (9 -> 7 -> 5 -> 3 -> 1),
//   then three linear heads 16 -> 11 scoring the offsets along z (dw), x (du) and y (dv).
// The proposal for a (voxel, atlas) pair is the 32 offsets of largest p_w * p_u * p_v.
constexpr int kCin = 2;
constexpr int kC = 16;
constexpr int kAxis = 11;            // offsets per axis (NH = 11)
constexpr int kHeads = 3 * kAxis;    // 33 logits
constexpr int kPatch = 9;
constexpr int kTopK = 32;            // proposals per (voxel, atlas)
constexpr float kInScale = 1.0f / 512.0f;  // MRI intensity scaling of the network input

// Flat parameter layout (float offsets).
constexpr int kW1 = 0;                                   // [16][2][27]
constexpr int kB1 = kW1 + kC * kCin * 27;                // [16]
constexpr int kW2 = kB1 + kC;                            // [16][16][27]
constexpr int kB2 = kW2 + kC * kC * 27;
constexpr int kW3 = kB2 + kC;
constexpr int kB3 = kW3 + kC * kC * 27;
constexpr int kW4 = kB3 + kC;
constexpr int kB4 = kW4 + kC * kC * 27;
constexpr int kH = kB4 + kC;                             // [33][16]
constexpr int kHB = kH + kHeads * kC;                    // [33]
constexpr int kParams = kHB + kHeads;                    // 22225

}  // namespace learned
}  // namespace pct
