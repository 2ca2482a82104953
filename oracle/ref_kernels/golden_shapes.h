// Shapes of the golden fixtures (tests/golden/golden_inputs.py holds the same numbers).
#pragma once
#define G_CAST_N (2ull * 4 * 64 * 2)
#define G_BF_A 20
#define G_BF_F 4
#define G_BF_T 256
#define G_BF_B 8
#define G_BF_TBLOCK 256
#define G_DET_A 2
#define G_DET_F 4
#define G_DET_T 512
#define G_DET_I 4
#define G_CH_A 2
#define G_CH_F 4
#define G_CH_T 256
