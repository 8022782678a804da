// layout.h - table layout shared by the host set-up and the kernels.
#pragma once

namespace cavity {

// Per-axis coefficient tables, `stride` entries each (n+1 used for face-indexed tables):
//   kW, kSp: width (cells) and spacing (faces); kInvW, kInvSp: their reciprocals;
//   kC3: weight of the wide (q = 3) Lamb stencil at a face; kInvNd3: 1 / distance of its nodes;
//   kEv1Lo/Hi, kEv3Lo/Hi: width-weighted interpolation to an edge from the narrow / wide stencil nodes;
//   kRamp: wall ramp of the 4th-order correction at a face index.
enum Tab : int { kW = 0, kSp, kInvW, kInvSp, kC3, kInvNd3, kEv1Lo, kEv1Hi, kEv3Lo, kEv3Hi, kRamp, kNumTabs };

}  // namespace cavity
