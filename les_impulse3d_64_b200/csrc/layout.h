// layout.h - table layout shared by the host set-up and the kernels.
#pragma once

namespace cavity {

// Per-axis coefficient tables, `stride` = n + 5 entries each, entry i + kTabOffset holding index i for
// i in [-2, n + 2] (zero where an index has no meaning):
//   kW, kSp: width (cells) and spacing (faces); kInvW, kInvSp: their reciprocals;
//   kC3: weight of the wide (q = 3) Lamb stencil at a face; kInvNd3: 1 / distance of its nodes;
//   kEv1Lo/Hi, kEv3Lo/Hi: width-weighted interpolation to an edge from the narrow / wide stencil nodes;
//   kRamp: wall ramp of the 4th-order correction at a face index;
//   kOk1, kOk3: 1 where the narrow / wide stencil around a face index lies inside the box, else 0;
//   kL1, kL3: kOk1 * kRamp, kOk3 * kRamp.
enum Tab : int { kW = 0, kSp, kInvW, kInvSp, kC3, kInvNd3, kEv1Lo, kEv1Hi, kEv3Lo, kEv3Hi, kRamp, kOk1, kOk3, kL1, kL3,
                 kNumTabs };
constexpr int kTabOffset = 2;
inline int tab_stride(int n) { return n + 5; }

}  // namespace cavity
