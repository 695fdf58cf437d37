// Parameter block of the edge-scoring MLP (FP32 masters, `TSPB_MLP_PARAMS` floats):
// W1[16][64] (rows >= 5 unused, kept zero), b1[64], W2[64][64], b2[64], w3[64], b3[1].
#pragma once

namespace tspb {

constexpr int MLP_F = 5;    // features per edge
constexpr int MLP_KX = 16;  // padded input width (one k-tile)
constexpr int MLP_H = 64;   // hidden width
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + MLP_KX * MLP_H;
constexpr int OFF_W2 = OFF_B1 + MLP_H;
constexpr int OFF_B2 = OFF_W2 + MLP_H * MLP_H;
constexpr int OFF_W3 = OFF_B2 + MLP_H;
constexpr int OFF_B3 = OFF_W3 + MLP_H;
constexpr int MLP_PARAMS = OFF_B3 + 1;

}  // namespace tspb
