// SCF choices per molecule-size bin of 32 AOs (bin k: 32k .. 32k+31 AOs, the
// last bin open), the defaults of ScfParams.  Written by the autotuner
// (python -m sparrow_b200.autotune); regenerate it after changing the SCF
// kernels.  Orbital update: 0 exact, 1 hybrid, 2 rotation.
//
// Measured on NVIDIA B200: SCF device ms of each bin's batch per candidate
// (orbital update / Pulay subspace), the chosen one marked *.
//   bin  0 (592 molecules): e/4 6.2, e/5 5.8, e/6 5.8, h/4 2.6*, h/5 2.6, h/6 2.6, r/4 2.8, r/5 2.8, r/6 3.0
//   bin  1 (592 molecules): e/4 15.3, e/5 14.6, e/6 14.2, h/4 5.4, h/5 5.4*, h/6 5.5, r/4 6.7, r/5 6.6, r/6 6.6
//   bin  2 (592 molecules): e/4 31.4, e/5 30.5, e/6 30.2, h/4 13.4, h/5 13.3*, h/6 13.4, r/4 19.5, r/5 19.2, r/6 19.4
//   bin  3 (592 molecules): e/4 50.9, e/5 50.0, e/6 48.9, h/4 22.9, h/5 22.6*, h/6 22.8, r/4 35.6, r/5 35.2, r/6 35.2
//   bin  4 (592 molecules): e/4 79.8, e/5 76.6, e/6 83.0, h/4 42.9, h/5 42.1*, h/6 42.7, r/4 71.0, r/5 70.3, r/6 70.3
//   bin  5 (592 molecules): e/4 124.1, e/5 121.7, e/6 116.2, h/4 61.4, h/5 60.7*, h/6 61.1, r/4 115.0, r/5 114.0, r/6 113.3
//   bin  6 (148 molecules): e/4 336.1, e/5 328.0, e/6 330.0, h/4 30.1, h/5 30.2, h/6 29.4*, r/4 158.4, r/5 157.8, r/6 159.0
//   bin  7 (148 molecules): e/4 120.2, e/5 114.2, e/6 114.3, h/4 37.5, h/5 36.9*, h/6 37.1, r/4 240.0, r/5 238.2, r/6 237.2
//   bin  8 (148 molecules): e/4 178.6, e/5 169.2, e/6 169.9, h/4 58.4, h/5 56.6*, h/6 56.9, r/4 349.7, r/5 348.8, r/6 346.7
//   bin  9 (148 molecules): e/4 229.9, e/5 407.4, e/6 410.5, h/4 70.5, h/5 68.8, h/6 68.7*, r/4 457.4, r/5 463.2(x), r/6 461.9
#pragma once
#define SGB_TUNED_ORBITAL_UPDATE {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1}
#define SGB_TUNED_DIIS_SIZE {4, 5, 5, 5, 5, 5, 6, 5, 5, 6, 6, 6, 6, 6, 6, 6}
