// GENERATED by gen_estimators.py -- do not edit by hand.
//
// Straight-line two-locus LD estimators for P = 1..4 populations (haplotype path).
// Statistic order and averaging weights follow moments.LD (pg_gpu ld_pipeline.py:357-457);
// raw-call algebra restates pg_gpu haplotype_kernels.py:69-304 in factored form.
#pragma once

#include "ldk_hap_feat.cuh"

// P = 1: 3 statistics from 3 distinct raw calls
template <typename T>
LDK_DEV void hap_features_P1(HapFeat<T>& x) {
    x.pA = x.c1 + x.c2;
    x.qA = x.c3 + x.c4;
    x.pB = x.c1 + x.c3;
    x.qB = x.c2 + x.c4;
    x.E = x.c1 * x.c4 - x.c2 * x.c3;
    x.a = x.qA - x.pA;
    x.b = x.qB - x.pB;
    x.s = (x.c2 + x.c3) - (x.c1 + x.c4);
    x.fA = x.pA * x.qA;
    x.fB = x.pB * x.qB;
    x.DDs = x.E * x.E - x.c1 * x.c4 * (x.c1 + x.c4 - T(1)) - x.c2 * x.c3 * (x.c2 + x.c3 - T(1));
    x.DZs = x.E * x.a * x.b + x.E * x.s + T(2) * (x.c2 * x.c3 + x.c1 * x.c4);
    x.PIs = x.fA * x.fB - x.c1 * x.c4 * (-T(1) + x.c1 + T(3) * x.c2 + T(3) * x.c3 + x.c4) - x.c2 * x.c3 * (-T(1) + T(3) * x.c1 + x.c2 + x.c3 + T(3) * x.c4);
}
template <typename T>
LDK_DEV void hap_stats_P1(const HapFeat<T>* f, T* acc) {
    const T v0 = f[0].DDs * f[0].r4;  // dd1(0,)
    const T v1 = f[0].DZs * f[0].r4;  // dz_iii(0,)
    const T v2 = f[0].PIs * f[0].r4;  // pi2_same(0,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // Dz_0_0_0
    acc[2] += v2;  // pi2_0_0_0_0
}

// P = 2: 15 statistics from 19 distinct raw calls
template <typename T>
LDK_DEV void hap_features_P2(HapFeat<T>& x) {
    x.pA = x.c1 + x.c2;
    x.qA = x.c3 + x.c4;
    x.pB = x.c1 + x.c3;
    x.qB = x.c2 + x.c4;
    x.E = x.c1 * x.c4 - x.c2 * x.c3;
    x.a = x.qA - x.pA;
    x.b = x.qB - x.pB;
    x.s = (x.c2 + x.c3) - (x.c1 + x.c4);
    x.fA = x.pA * x.qA;
    x.fB = x.pB * x.qB;
    x.Q1 = x.c1 * (T(1) - x.ns + x.c4) - x.c2 * x.c3;
    x.Q2 = x.c2 * (T(1) - x.ns + x.c3) - x.c1 * x.c4;
    x.Q3 = x.c3 * (T(1) - x.ns + x.c2) - x.c1 * x.c4;
    x.Q4 = x.c4 * (T(1) - x.ns + x.c1) - x.c2 * x.c3;
    x.L1 = x.c4 * (x.ns - x.c1) + x.c2 * x.c3;
    x.L2 = x.c3 * (x.ns - x.c2) + x.c1 * x.c4;
    x.L3 = x.c2 * (x.ns - x.c3) + x.c1 * x.c4;
    x.L4 = x.c1 * (x.ns - x.c4) + x.c2 * x.c3;
    x.T1 = x.fA * x.qB - x.c1 * x.c4 - x.c2 * x.c3 - T(2) * x.c2 * x.c4;
    x.T2 = x.fA * x.pB - T(2) * x.c1 * x.c3 - x.c1 * x.c4 - x.c2 * x.c3;
    x.DDs = x.E * x.E - x.c1 * x.c4 * (x.c1 + x.c4 - T(1)) - x.c2 * x.c3 * (x.c2 + x.c3 - T(1));
    x.DZs = x.E * x.a * x.b + x.E * x.s + T(2) * (x.c2 * x.c3 + x.c1 * x.c4);
    x.PIs = x.fA * x.fB - x.c1 * x.c4 * (-T(1) + x.c1 + T(3) * x.c2 + T(3) * x.c3 + x.c4) - x.c2 * x.c3 * (-T(1) + T(3) * x.c1 + x.c2 + x.c3 + T(3) * x.c4);
}
template <typename T>
LDK_DEV void hap_stats_P2(const HapFeat<T>* f, T* acc) {
    const T v0 = f[0].DDs * f[0].r4;  // dd1(0,)
    const T v1 = (f[0].E * f[1].E) * (f[0].r2 * f[1].r2);  // dd2(0, 1)
    const T v2 = f[1].DDs * f[1].r4;  // dd1(1,)
    const T v3 = f[0].DZs * f[0].r4;  // dz_iii(0,)
    const T v4 = (f[0].a * f[0].E * f[1].b) * (f[0].r3 * f[1].r1);  // dz_iij(0, 1)
    const T v5 = (f[0].b * f[0].E * f[1].a) * (f[0].r3 * f[1].r1);  // dz_iji(0, 1)
    const T v6 = (f[0].E * (f[1].s + f[1].b * f[1].a)) * (f[0].r2 * f[1].r2);  // dz_ijj(0, 1)
    const T v7 = (f[1].E * (f[0].s + f[0].b * f[0].a)) * (f[1].r2 * f[0].r2);  // dz_ijj(1, 0)
    const T v8 = (f[1].b * f[1].E * f[0].a) * (f[1].r3 * f[0].r1);  // dz_iji(1, 0)
    const T v9 = (f[1].a * f[1].E * f[0].b) * (f[1].r3 * f[0].r1);  // dz_iij(1, 0)
    const T v10 = f[1].DZs * f[1].r4;  // dz_iii(1,)
    const T v11 = f[0].PIs * f[0].r4;  // pi2_same(0,)
    const T v12 = T(0.5) * (f[1].pB * f[0].T1 + f[1].qB * f[0].T2) * (f[0].r3 * f[1].r1);  // pi2_triple(0, 1)
    const T v13 = (f[0].fA * f[1].fB) * (f[0].r2 * f[1].r2);  // pi2_iikk(0, 1)
    const T v14 = (f[1].fA * f[0].fB) * (f[1].r2 * f[0].r2);  // pi2_iikk(1, 0)
    const T v15 = T(0.25) * ((f[0].pA * f[1].qA + f[0].qA * f[1].pA) * (f[0].pB * f[1].qB + f[0].qB * f[1].pB) + (f[0].Q1 * f[1].c4 + f[0].Q2 * f[1].c3 + f[0].Q3 * f[1].c2 + f[0].Q4 * f[1].c1 - (f[0].c1 * f[1].L1 + f[0].c2 * f[1].L2 + f[0].c3 * f[1].L3 + f[0].c4 * f[1].L4))) * (f[0].r2 * f[1].r2);  // pi2_ijij(0, 1)
    const T v16 = T(0.25) * ((f[1].pA * f[0].qA + f[1].qA * f[0].pA) * (f[1].pB * f[0].qB + f[1].qB * f[0].pB) + (f[1].Q1 * f[0].c4 + f[1].Q2 * f[0].c3 + f[1].Q3 * f[0].c2 + f[1].Q4 * f[0].c1 - (f[1].c1 * f[0].L1 + f[1].c2 * f[0].L2 + f[1].c3 * f[0].L3 + f[1].c4 * f[0].L4))) * (f[1].r2 * f[0].r2);  // pi2_ijij(1, 0)
    const T v17 = T(0.5) * (f[0].pB * f[1].T1 + f[0].qB * f[1].T2) * (f[1].r3 * f[0].r1);  // pi2_triple(1, 0)
    const T v18 = f[1].PIs * f[1].r4;  // pi2_same(1,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // DD_0_1
    acc[2] += v2;  // DD_1_1
    acc[3] += v3;  // Dz_0_0_0
    acc[4] += T(0.5) * (v4 + v5);  // Dz_0_0_1
    acc[5] += v6;  // Dz_0_1_1
    acc[6] += v7;  // Dz_1_0_0
    acc[7] += T(0.5) * (v8 + v9);  // Dz_1_0_1
    acc[8] += v10;  // Dz_1_1_1
    acc[9] += v11;  // pi2_0_0_0_0
    acc[10] += v12;  // pi2_0_0_0_1
    acc[11] += T(0.5) * (v13 + v14);  // pi2_0_0_1_1
    acc[12] += T(0.5) * (v15 + v16);  // pi2_0_1_0_1
    acc[13] += v17;  // pi2_0_1_1_1
    acc[14] += v18;  // pi2_1_1_1_1
}

// P = 3: 45 statistics from 66 distinct raw calls
template <typename T>
LDK_DEV void hap_features_P3(HapFeat<T>& x) {
    x.pA = x.c1 + x.c2;
    x.qA = x.c3 + x.c4;
    x.pB = x.c1 + x.c3;
    x.qB = x.c2 + x.c4;
    x.E = x.c1 * x.c4 - x.c2 * x.c3;
    x.a = x.qA - x.pA;
    x.b = x.qB - x.pB;
    x.s = (x.c2 + x.c3) - (x.c1 + x.c4);
    x.fA = x.pA * x.qA;
    x.fB = x.pB * x.qB;
    x.Q1 = x.c1 * (T(1) - x.ns + x.c4) - x.c2 * x.c3;
    x.Q2 = x.c2 * (T(1) - x.ns + x.c3) - x.c1 * x.c4;
    x.Q3 = x.c3 * (T(1) - x.ns + x.c2) - x.c1 * x.c4;
    x.Q4 = x.c4 * (T(1) - x.ns + x.c1) - x.c2 * x.c3;
    x.L1 = x.c4 * (x.ns - x.c1) + x.c2 * x.c3;
    x.L2 = x.c3 * (x.ns - x.c2) + x.c1 * x.c4;
    x.L3 = x.c2 * (x.ns - x.c3) + x.c1 * x.c4;
    x.L4 = x.c1 * (x.ns - x.c4) + x.c2 * x.c3;
    x.T1 = x.fA * x.qB - x.c1 * x.c4 - x.c2 * x.c3 - T(2) * x.c2 * x.c4;
    x.T2 = x.fA * x.pB - T(2) * x.c1 * x.c3 - x.c1 * x.c4 - x.c2 * x.c3;
    x.DDs = x.E * x.E - x.c1 * x.c4 * (x.c1 + x.c4 - T(1)) - x.c2 * x.c3 * (x.c2 + x.c3 - T(1));
    x.DZs = x.E * x.a * x.b + x.E * x.s + T(2) * (x.c2 * x.c3 + x.c1 * x.c4);
    x.PIs = x.fA * x.fB - x.c1 * x.c4 * (-T(1) + x.c1 + T(3) * x.c2 + T(3) * x.c3 + x.c4) - x.c2 * x.c3 * (-T(1) + T(3) * x.c1 + x.c2 + x.c3 + T(3) * x.c4);
}
template <typename T>
LDK_DEV void hap_stats_P3(const HapFeat<T>* f, T* acc) {
    const T v0 = f[0].DDs * f[0].r4;  // dd1(0,)
    const T v1 = (f[0].E * f[1].E) * (f[0].r2 * f[1].r2);  // dd2(0, 1)
    const T v2 = (f[0].E * f[2].E) * (f[0].r2 * f[2].r2);  // dd2(0, 2)
    const T v3 = f[1].DDs * f[1].r4;  // dd1(1,)
    const T v4 = (f[1].E * f[2].E) * (f[1].r2 * f[2].r2);  // dd2(1, 2)
    const T v5 = f[2].DDs * f[2].r4;  // dd1(2,)
    const T v6 = f[0].DZs * f[0].r4;  // dz_iii(0,)
    const T v7 = (f[0].a * f[0].E * f[1].b) * (f[0].r3 * f[1].r1);  // dz_iij(0, 1)
    const T v8 = (f[0].b * f[0].E * f[1].a) * (f[0].r3 * f[1].r1);  // dz_iji(0, 1)
    const T v9 = (f[0].a * f[0].E * f[2].b) * (f[0].r3 * f[2].r1);  // dz_iij(0, 2)
    const T v10 = (f[0].b * f[0].E * f[2].a) * (f[0].r3 * f[2].r1);  // dz_iji(0, 2)
    const T v11 = (f[0].E * (f[1].s + f[1].b * f[1].a)) * (f[0].r2 * f[1].r2);  // dz_ijj(0, 1)
    const T v12 = (f[0].E * f[1].a * f[2].b) * (f[0].r2 * f[1].r1 * f[2].r1);  // dz_ijk(0, 1, 2)
    const T v13 = (f[0].E * f[2].a * f[1].b) * (f[0].r2 * f[2].r1 * f[1].r1);  // dz_ijk(0, 2, 1)
    const T v14 = (f[0].E * (f[2].s + f[2].b * f[2].a)) * (f[0].r2 * f[2].r2);  // dz_ijj(0, 2)
    const T v15 = (f[1].E * (f[0].s + f[0].b * f[0].a)) * (f[1].r2 * f[0].r2);  // dz_ijj(1, 0)
    const T v16 = (f[1].b * f[1].E * f[0].a) * (f[1].r3 * f[0].r1);  // dz_iji(1, 0)
    const T v17 = (f[1].a * f[1].E * f[0].b) * (f[1].r3 * f[0].r1);  // dz_iij(1, 0)
    const T v18 = (f[1].E * f[0].a * f[2].b) * (f[1].r2 * f[0].r1 * f[2].r1);  // dz_ijk(1, 0, 2)
    const T v19 = (f[1].E * f[2].a * f[0].b) * (f[1].r2 * f[2].r1 * f[0].r1);  // dz_ijk(1, 2, 0)
    const T v20 = f[1].DZs * f[1].r4;  // dz_iii(1,)
    const T v21 = (f[1].a * f[1].E * f[2].b) * (f[1].r3 * f[2].r1);  // dz_iij(1, 2)
    const T v22 = (f[1].b * f[1].E * f[2].a) * (f[1].r3 * f[2].r1);  // dz_iji(1, 2)
    const T v23 = (f[1].E * (f[2].s + f[2].b * f[2].a)) * (f[1].r2 * f[2].r2);  // dz_ijj(1, 2)
    const T v24 = (f[2].E * (f[0].s + f[0].b * f[0].a)) * (f[2].r2 * f[0].r2);  // dz_ijj(2, 0)
    const T v25 = (f[2].E * f[0].a * f[1].b) * (f[2].r2 * f[0].r1 * f[1].r1);  // dz_ijk(2, 0, 1)
    const T v26 = (f[2].E * f[1].a * f[0].b) * (f[2].r2 * f[1].r1 * f[0].r1);  // dz_ijk(2, 1, 0)
    const T v27 = (f[2].b * f[2].E * f[0].a) * (f[2].r3 * f[0].r1);  // dz_iji(2, 0)
    const T v28 = (f[2].a * f[2].E * f[0].b) * (f[2].r3 * f[0].r1);  // dz_iij(2, 0)
    const T v29 = (f[2].E * (f[1].s + f[1].b * f[1].a)) * (f[2].r2 * f[1].r2);  // dz_ijj(2, 1)
    const T v30 = (f[2].b * f[2].E * f[1].a) * (f[2].r3 * f[1].r1);  // dz_iji(2, 1)
    const T v31 = (f[2].a * f[2].E * f[1].b) * (f[2].r3 * f[1].r1);  // dz_iij(2, 1)
    const T v32 = f[2].DZs * f[2].r4;  // dz_iii(2,)
    const T v33 = f[0].PIs * f[0].r4;  // pi2_same(0,)
    const T v34 = T(0.5) * (f[1].pB * f[0].T1 + f[1].qB * f[0].T2) * (f[0].r3 * f[1].r1);  // pi2_triple(0, 1)
    const T v35 = T(0.5) * (f[2].pB * f[0].T1 + f[2].qB * f[0].T2) * (f[0].r3 * f[2].r1);  // pi2_triple(0, 2)
    const T v36 = (f[0].fA * f[1].fB) * (f[0].r2 * f[1].r2);  // pi2_iikk(0, 1)
    const T v37 = (f[1].fA * f[0].fB) * (f[1].r2 * f[0].r2);  // pi2_iikk(1, 0)
    const T v38 = T(0.5) * (f[0].fA * (f[1].pB * f[2].qB + f[1].qB * f[2].pB)) * (f[0].r2 * f[1].r1 * f[2].r1);  // pi2_iikl(0, 1, 2)
    const T v39 = T(0.5) * (f[0].fB * (f[1].pA * f[2].qA + f[1].qA * f[2].pA)) * (f[0].r2 * f[1].r1 * f[2].r1);  // pi2_ijkk(1, 2, 0)
    const T v40 = (f[0].fA * f[2].fB) * (f[0].r2 * f[2].r2);  // pi2_iikk(0, 2)
    const T v41 = (f[2].fA * f[0].fB) * (f[2].r2 * f[0].r2);  // pi2_iikk(2, 0)
    const T v42 = T(0.25) * ((f[0].pA * f[1].qA + f[0].qA * f[1].pA) * (f[0].pB * f[1].qB + f[0].qB * f[1].pB) + (f[0].Q1 * f[1].c4 + f[0].Q2 * f[1].c3 + f[0].Q3 * f[1].c2 + f[0].Q4 * f[1].c1 - (f[0].c1 * f[1].L1 + f[0].c2 * f[1].L2 + f[0].c3 * f[1].L3 + f[0].c4 * f[1].L4))) * (f[0].r2 * f[1].r2);  // pi2_ijij(0, 1)
    const T v43 = T(0.25) * ((f[1].pA * f[0].qA + f[1].qA * f[0].pA) * (f[1].pB * f[0].qB + f[1].qB * f[0].pB) + (f[1].Q1 * f[0].c4 + f[1].Q2 * f[0].c3 + f[1].Q3 * f[0].c2 + f[1].Q4 * f[0].c1 - (f[1].c1 * f[0].L1 + f[1].c2 * f[0].L2 + f[1].c3 * f[0].L3 + f[1].c4 * f[0].L4))) * (f[1].r2 * f[0].r2);  // pi2_ijij(1, 0)
    const T v44 = T(0.25) * (f[1].pA * (f[2].pB * (f[0].L1 - f[0].c4) + f[2].qB * (f[0].L2 - f[0].c3)) + f[1].qA * (f[2].pB * (f[0].L3 - f[0].c2) + f[2].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[1].r1 * f[2].r1);  // pi2_shared(0, 1, 2)
    const T v45 = T(0.25) * (f[2].pA * (f[1].pB * (f[0].L1 - f[0].c4) + f[1].qB * (f[0].L2 - f[0].c3)) + f[2].qA * (f[1].pB * (f[0].L3 - f[0].c2) + f[1].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[2].r1 * f[1].r1);  // pi2_shared(0, 2, 1)
    const T v46 = T(0.5) * (f[0].pB * f[1].T1 + f[0].qB * f[1].T2) * (f[1].r3 * f[0].r1);  // pi2_triple(1, 0)
    const T v47 = T(0.25) * (f[0].pA * (f[2].pB * (f[1].L1 - f[1].c4) + f[2].qB * (f[1].L2 - f[1].c3)) + f[0].qA * (f[2].pB * (f[1].L3 - f[1].c2) + f[2].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[0].r1 * f[2].r1);  // pi2_shared(1, 0, 2)
    const T v48 = T(0.25) * (f[2].pA * (f[0].pB * (f[1].L1 - f[1].c4) + f[0].qB * (f[1].L2 - f[1].c3)) + f[2].qA * (f[0].pB * (f[1].L3 - f[1].c2) + f[0].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[2].r1 * f[0].r1);  // pi2_shared(1, 2, 0)
    const T v49 = T(0.5) * (f[2].fB * (f[0].pA * f[1].qA + f[0].qA * f[1].pA)) * (f[2].r2 * f[0].r1 * f[1].r1);  // pi2_ijkk(0, 1, 2)
    const T v50 = T(0.5) * (f[2].fA * (f[0].pB * f[1].qB + f[0].qB * f[1].pB)) * (f[2].r2 * f[0].r1 * f[1].r1);  // pi2_iikl(2, 0, 1)
    const T v51 = T(0.25) * ((f[0].pA * f[2].qA + f[0].qA * f[2].pA) * (f[0].pB * f[2].qB + f[0].qB * f[2].pB) + (f[0].Q1 * f[2].c4 + f[0].Q2 * f[2].c3 + f[0].Q3 * f[2].c2 + f[0].Q4 * f[2].c1 - (f[0].c1 * f[2].L1 + f[0].c2 * f[2].L2 + f[0].c3 * f[2].L3 + f[0].c4 * f[2].L4))) * (f[0].r2 * f[2].r2);  // pi2_ijij(0, 2)
    const T v52 = T(0.25) * ((f[2].pA * f[0].qA + f[2].qA * f[0].pA) * (f[2].pB * f[0].qB + f[2].qB * f[0].pB) + (f[2].Q1 * f[0].c4 + f[2].Q2 * f[0].c3 + f[2].Q3 * f[0].c2 + f[2].Q4 * f[0].c1 - (f[2].c1 * f[0].L1 + f[2].c2 * f[0].L2 + f[2].c3 * f[0].L3 + f[2].c4 * f[0].L4))) * (f[2].r2 * f[0].r2);  // pi2_ijij(2, 0)
    const T v53 = T(0.5) * (f[1].fB * (f[0].pA * f[2].qA + f[0].qA * f[2].pA)) * (f[1].r2 * f[0].r1 * f[2].r1);  // pi2_ijkk(0, 2, 1)
    const T v54 = T(0.5) * (f[1].fA * (f[0].pB * f[2].qB + f[0].qB * f[2].pB)) * (f[1].r2 * f[0].r1 * f[2].r1);  // pi2_iikl(1, 0, 2)
    const T v55 = T(0.25) * (f[0].pA * (f[1].pB * (f[2].L1 - f[2].c4) + f[1].qB * (f[2].L2 - f[2].c3)) + f[0].qA * (f[1].pB * (f[2].L3 - f[2].c2) + f[1].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[0].r1 * f[1].r1);  // pi2_shared(2, 0, 1)
    const T v56 = T(0.25) * (f[1].pA * (f[0].pB * (f[2].L1 - f[2].c4) + f[0].qB * (f[2].L2 - f[2].c3)) + f[1].qA * (f[0].pB * (f[2].L3 - f[2].c2) + f[0].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[1].r1 * f[0].r1);  // pi2_shared(2, 1, 0)
    const T v57 = T(0.5) * (f[0].pB * f[2].T1 + f[0].qB * f[2].T2) * (f[2].r3 * f[0].r1);  // pi2_triple(2, 0)
    const T v58 = f[1].PIs * f[1].r4;  // pi2_same(1,)
    const T v59 = T(0.5) * (f[2].pB * f[1].T1 + f[2].qB * f[1].T2) * (f[1].r3 * f[2].r1);  // pi2_triple(1, 2)
    const T v60 = (f[1].fA * f[2].fB) * (f[1].r2 * f[2].r2);  // pi2_iikk(1, 2)
    const T v61 = (f[2].fA * f[1].fB) * (f[2].r2 * f[1].r2);  // pi2_iikk(2, 1)
    const T v62 = T(0.25) * ((f[1].pA * f[2].qA + f[1].qA * f[2].pA) * (f[1].pB * f[2].qB + f[1].qB * f[2].pB) + (f[1].Q1 * f[2].c4 + f[1].Q2 * f[2].c3 + f[1].Q3 * f[2].c2 + f[1].Q4 * f[2].c1 - (f[1].c1 * f[2].L1 + f[1].c2 * f[2].L2 + f[1].c3 * f[2].L3 + f[1].c4 * f[2].L4))) * (f[1].r2 * f[2].r2);  // pi2_ijij(1, 2)
    const T v63 = T(0.25) * ((f[2].pA * f[1].qA + f[2].qA * f[1].pA) * (f[2].pB * f[1].qB + f[2].qB * f[1].pB) + (f[2].Q1 * f[1].c4 + f[2].Q2 * f[1].c3 + f[2].Q3 * f[1].c2 + f[2].Q4 * f[1].c1 - (f[2].c1 * f[1].L1 + f[2].c2 * f[1].L2 + f[2].c3 * f[1].L3 + f[2].c4 * f[1].L4))) * (f[2].r2 * f[1].r2);  // pi2_ijij(2, 1)
    const T v64 = T(0.5) * (f[1].pB * f[2].T1 + f[1].qB * f[2].T2) * (f[2].r3 * f[1].r1);  // pi2_triple(2, 1)
    const T v65 = f[2].PIs * f[2].r4;  // pi2_same(2,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // DD_0_1
    acc[2] += v2;  // DD_0_2
    acc[3] += v3;  // DD_1_1
    acc[4] += v4;  // DD_1_2
    acc[5] += v5;  // DD_2_2
    acc[6] += v6;  // Dz_0_0_0
    acc[7] += T(0.5) * (v7 + v8);  // Dz_0_0_1
    acc[8] += T(0.5) * (v9 + v10);  // Dz_0_0_2
    acc[9] += v11;  // Dz_0_1_1
    acc[10] += T(0.5) * (v12 + v13);  // Dz_0_1_2
    acc[11] += v14;  // Dz_0_2_2
    acc[12] += v15;  // Dz_1_0_0
    acc[13] += T(0.5) * (v16 + v17);  // Dz_1_0_1
    acc[14] += T(0.5) * (v18 + v19);  // Dz_1_0_2
    acc[15] += v20;  // Dz_1_1_1
    acc[16] += T(0.5) * (v21 + v22);  // Dz_1_1_2
    acc[17] += v23;  // Dz_1_2_2
    acc[18] += v24;  // Dz_2_0_0
    acc[19] += T(0.5) * (v25 + v26);  // Dz_2_0_1
    acc[20] += T(0.5) * (v27 + v28);  // Dz_2_0_2
    acc[21] += v29;  // Dz_2_1_1
    acc[22] += T(0.5) * (v30 + v31);  // Dz_2_1_2
    acc[23] += v32;  // Dz_2_2_2
    acc[24] += v33;  // pi2_0_0_0_0
    acc[25] += v34;  // pi2_0_0_0_1
    acc[26] += v35;  // pi2_0_0_0_2
    acc[27] += T(0.5) * (v36 + v37);  // pi2_0_0_1_1
    acc[28] += T(0.5) * (v38 + v39);  // pi2_0_0_1_2
    acc[29] += T(0.5) * (v40 + v41);  // pi2_0_0_2_2
    acc[30] += T(0.5) * (v42 + v43);  // pi2_0_1_0_1
    acc[31] += T(0.5) * (v44 + v45);  // pi2_0_1_0_2
    acc[32] += v46;  // pi2_0_1_1_1
    acc[33] += T(0.5) * (v47 + v48);  // pi2_0_1_1_2
    acc[34] += T(0.5) * (v49 + v50);  // pi2_0_1_2_2
    acc[35] += T(0.5) * (v51 + v52);  // pi2_0_2_0_2
    acc[36] += T(0.5) * (v53 + v54);  // pi2_0_2_1_1
    acc[37] += T(0.5) * (v55 + v56);  // pi2_0_2_1_2
    acc[38] += v57;  // pi2_0_2_2_2
    acc[39] += v58;  // pi2_1_1_1_1
    acc[40] += v59;  // pi2_1_1_1_2
    acc[41] += T(0.5) * (v60 + v61);  // pi2_1_1_2_2
    acc[42] += T(0.5) * (v62 + v63);  // pi2_1_2_1_2
    acc[43] += v64;  // pi2_1_2_2_2
    acc[44] += v65;  // pi2_2_2_2_2
}

// P = 4: 105 statistics from 168 distinct raw calls
template <typename T>
LDK_DEV void hap_features_P4(HapFeat<T>& x) {
    x.pA = x.c1 + x.c2;
    x.qA = x.c3 + x.c4;
    x.pB = x.c1 + x.c3;
    x.qB = x.c2 + x.c4;
    x.E = x.c1 * x.c4 - x.c2 * x.c3;
    x.a = x.qA - x.pA;
    x.b = x.qB - x.pB;
    x.s = (x.c2 + x.c3) - (x.c1 + x.c4);
    x.fA = x.pA * x.qA;
    x.fB = x.pB * x.qB;
    x.Q1 = x.c1 * (T(1) - x.ns + x.c4) - x.c2 * x.c3;
    x.Q2 = x.c2 * (T(1) - x.ns + x.c3) - x.c1 * x.c4;
    x.Q3 = x.c3 * (T(1) - x.ns + x.c2) - x.c1 * x.c4;
    x.Q4 = x.c4 * (T(1) - x.ns + x.c1) - x.c2 * x.c3;
    x.L1 = x.c4 * (x.ns - x.c1) + x.c2 * x.c3;
    x.L2 = x.c3 * (x.ns - x.c2) + x.c1 * x.c4;
    x.L3 = x.c2 * (x.ns - x.c3) + x.c1 * x.c4;
    x.L4 = x.c1 * (x.ns - x.c4) + x.c2 * x.c3;
    x.T1 = x.fA * x.qB - x.c1 * x.c4 - x.c2 * x.c3 - T(2) * x.c2 * x.c4;
    x.T2 = x.fA * x.pB - T(2) * x.c1 * x.c3 - x.c1 * x.c4 - x.c2 * x.c3;
    x.DDs = x.E * x.E - x.c1 * x.c4 * (x.c1 + x.c4 - T(1)) - x.c2 * x.c3 * (x.c2 + x.c3 - T(1));
    x.DZs = x.E * x.a * x.b + x.E * x.s + T(2) * (x.c2 * x.c3 + x.c1 * x.c4);
    x.PIs = x.fA * x.fB - x.c1 * x.c4 * (-T(1) + x.c1 + T(3) * x.c2 + T(3) * x.c3 + x.c4) - x.c2 * x.c3 * (-T(1) + T(3) * x.c1 + x.c2 + x.c3 + T(3) * x.c4);
}
template <typename T>
LDK_DEV void hap_stats_P4(const HapFeat<T>* f, T* acc) {
    const T v0 = f[0].DDs * f[0].r4;  // dd1(0,)
    const T v1 = (f[0].E * f[1].E) * (f[0].r2 * f[1].r2);  // dd2(0, 1)
    const T v2 = (f[0].E * f[2].E) * (f[0].r2 * f[2].r2);  // dd2(0, 2)
    const T v3 = (f[0].E * f[3].E) * (f[0].r2 * f[3].r2);  // dd2(0, 3)
    const T v4 = f[1].DDs * f[1].r4;  // dd1(1,)
    const T v5 = (f[1].E * f[2].E) * (f[1].r2 * f[2].r2);  // dd2(1, 2)
    const T v6 = (f[1].E * f[3].E) * (f[1].r2 * f[3].r2);  // dd2(1, 3)
    const T v7 = f[2].DDs * f[2].r4;  // dd1(2,)
    const T v8 = (f[2].E * f[3].E) * (f[2].r2 * f[3].r2);  // dd2(2, 3)
    const T v9 = f[3].DDs * f[3].r4;  // dd1(3,)
    const T v10 = f[0].DZs * f[0].r4;  // dz_iii(0,)
    const T v11 = (f[0].a * f[0].E * f[1].b) * (f[0].r3 * f[1].r1);  // dz_iij(0, 1)
    const T v12 = (f[0].b * f[0].E * f[1].a) * (f[0].r3 * f[1].r1);  // dz_iji(0, 1)
    const T v13 = (f[0].a * f[0].E * f[2].b) * (f[0].r3 * f[2].r1);  // dz_iij(0, 2)
    const T v14 = (f[0].b * f[0].E * f[2].a) * (f[0].r3 * f[2].r1);  // dz_iji(0, 2)
    const T v15 = (f[0].a * f[0].E * f[3].b) * (f[0].r3 * f[3].r1);  // dz_iij(0, 3)
    const T v16 = (f[0].b * f[0].E * f[3].a) * (f[0].r3 * f[3].r1);  // dz_iji(0, 3)
    const T v17 = (f[0].E * (f[1].s + f[1].b * f[1].a)) * (f[0].r2 * f[1].r2);  // dz_ijj(0, 1)
    const T v18 = (f[0].E * f[1].a * f[2].b) * (f[0].r2 * f[1].r1 * f[2].r1);  // dz_ijk(0, 1, 2)
    const T v19 = (f[0].E * f[2].a * f[1].b) * (f[0].r2 * f[2].r1 * f[1].r1);  // dz_ijk(0, 2, 1)
    const T v20 = (f[0].E * f[1].a * f[3].b) * (f[0].r2 * f[1].r1 * f[3].r1);  // dz_ijk(0, 1, 3)
    const T v21 = (f[0].E * f[3].a * f[1].b) * (f[0].r2 * f[3].r1 * f[1].r1);  // dz_ijk(0, 3, 1)
    const T v22 = (f[0].E * (f[2].s + f[2].b * f[2].a)) * (f[0].r2 * f[2].r2);  // dz_ijj(0, 2)
    const T v23 = (f[0].E * f[2].a * f[3].b) * (f[0].r2 * f[2].r1 * f[3].r1);  // dz_ijk(0, 2, 3)
    const T v24 = (f[0].E * f[3].a * f[2].b) * (f[0].r2 * f[3].r1 * f[2].r1);  // dz_ijk(0, 3, 2)
    const T v25 = (f[0].E * (f[3].s + f[3].b * f[3].a)) * (f[0].r2 * f[3].r2);  // dz_ijj(0, 3)
    const T v26 = (f[1].E * (f[0].s + f[0].b * f[0].a)) * (f[1].r2 * f[0].r2);  // dz_ijj(1, 0)
    const T v27 = (f[1].b * f[1].E * f[0].a) * (f[1].r3 * f[0].r1);  // dz_iji(1, 0)
    const T v28 = (f[1].a * f[1].E * f[0].b) * (f[1].r3 * f[0].r1);  // dz_iij(1, 0)
    const T v29 = (f[1].E * f[0].a * f[2].b) * (f[1].r2 * f[0].r1 * f[2].r1);  // dz_ijk(1, 0, 2)
    const T v30 = (f[1].E * f[2].a * f[0].b) * (f[1].r2 * f[2].r1 * f[0].r1);  // dz_ijk(1, 2, 0)
    const T v31 = (f[1].E * f[0].a * f[3].b) * (f[1].r2 * f[0].r1 * f[3].r1);  // dz_ijk(1, 0, 3)
    const T v32 = (f[1].E * f[3].a * f[0].b) * (f[1].r2 * f[3].r1 * f[0].r1);  // dz_ijk(1, 3, 0)
    const T v33 = f[1].DZs * f[1].r4;  // dz_iii(1,)
    const T v34 = (f[1].a * f[1].E * f[2].b) * (f[1].r3 * f[2].r1);  // dz_iij(1, 2)
    const T v35 = (f[1].b * f[1].E * f[2].a) * (f[1].r3 * f[2].r1);  // dz_iji(1, 2)
    const T v36 = (f[1].a * f[1].E * f[3].b) * (f[1].r3 * f[3].r1);  // dz_iij(1, 3)
    const T v37 = (f[1].b * f[1].E * f[3].a) * (f[1].r3 * f[3].r1);  // dz_iji(1, 3)
    const T v38 = (f[1].E * (f[2].s + f[2].b * f[2].a)) * (f[1].r2 * f[2].r2);  // dz_ijj(1, 2)
    const T v39 = (f[1].E * f[2].a * f[3].b) * (f[1].r2 * f[2].r1 * f[3].r1);  // dz_ijk(1, 2, 3)
    const T v40 = (f[1].E * f[3].a * f[2].b) * (f[1].r2 * f[3].r1 * f[2].r1);  // dz_ijk(1, 3, 2)
    const T v41 = (f[1].E * (f[3].s + f[3].b * f[3].a)) * (f[1].r2 * f[3].r2);  // dz_ijj(1, 3)
    const T v42 = (f[2].E * (f[0].s + f[0].b * f[0].a)) * (f[2].r2 * f[0].r2);  // dz_ijj(2, 0)
    const T v43 = (f[2].E * f[0].a * f[1].b) * (f[2].r2 * f[0].r1 * f[1].r1);  // dz_ijk(2, 0, 1)
    const T v44 = (f[2].E * f[1].a * f[0].b) * (f[2].r2 * f[1].r1 * f[0].r1);  // dz_ijk(2, 1, 0)
    const T v45 = (f[2].b * f[2].E * f[0].a) * (f[2].r3 * f[0].r1);  // dz_iji(2, 0)
    const T v46 = (f[2].a * f[2].E * f[0].b) * (f[2].r3 * f[0].r1);  // dz_iij(2, 0)
    const T v47 = (f[2].E * f[0].a * f[3].b) * (f[2].r2 * f[0].r1 * f[3].r1);  // dz_ijk(2, 0, 3)
    const T v48 = (f[2].E * f[3].a * f[0].b) * (f[2].r2 * f[3].r1 * f[0].r1);  // dz_ijk(2, 3, 0)
    const T v49 = (f[2].E * (f[1].s + f[1].b * f[1].a)) * (f[2].r2 * f[1].r2);  // dz_ijj(2, 1)
    const T v50 = (f[2].b * f[2].E * f[1].a) * (f[2].r3 * f[1].r1);  // dz_iji(2, 1)
    const T v51 = (f[2].a * f[2].E * f[1].b) * (f[2].r3 * f[1].r1);  // dz_iij(2, 1)
    const T v52 = (f[2].E * f[1].a * f[3].b) * (f[2].r2 * f[1].r1 * f[3].r1);  // dz_ijk(2, 1, 3)
    const T v53 = (f[2].E * f[3].a * f[1].b) * (f[2].r2 * f[3].r1 * f[1].r1);  // dz_ijk(2, 3, 1)
    const T v54 = f[2].DZs * f[2].r4;  // dz_iii(2,)
    const T v55 = (f[2].a * f[2].E * f[3].b) * (f[2].r3 * f[3].r1);  // dz_iij(2, 3)
    const T v56 = (f[2].b * f[2].E * f[3].a) * (f[2].r3 * f[3].r1);  // dz_iji(2, 3)
    const T v57 = (f[2].E * (f[3].s + f[3].b * f[3].a)) * (f[2].r2 * f[3].r2);  // dz_ijj(2, 3)
    const T v58 = (f[3].E * (f[0].s + f[0].b * f[0].a)) * (f[3].r2 * f[0].r2);  // dz_ijj(3, 0)
    const T v59 = (f[3].E * f[0].a * f[1].b) * (f[3].r2 * f[0].r1 * f[1].r1);  // dz_ijk(3, 0, 1)
    const T v60 = (f[3].E * f[1].a * f[0].b) * (f[3].r2 * f[1].r1 * f[0].r1);  // dz_ijk(3, 1, 0)
    const T v61 = (f[3].E * f[0].a * f[2].b) * (f[3].r2 * f[0].r1 * f[2].r1);  // dz_ijk(3, 0, 2)
    const T v62 = (f[3].E * f[2].a * f[0].b) * (f[3].r2 * f[2].r1 * f[0].r1);  // dz_ijk(3, 2, 0)
    const T v63 = (f[3].b * f[3].E * f[0].a) * (f[3].r3 * f[0].r1);  // dz_iji(3, 0)
    const T v64 = (f[3].a * f[3].E * f[0].b) * (f[3].r3 * f[0].r1);  // dz_iij(3, 0)
    const T v65 = (f[3].E * (f[1].s + f[1].b * f[1].a)) * (f[3].r2 * f[1].r2);  // dz_ijj(3, 1)
    const T v66 = (f[3].E * f[1].a * f[2].b) * (f[3].r2 * f[1].r1 * f[2].r1);  // dz_ijk(3, 1, 2)
    const T v67 = (f[3].E * f[2].a * f[1].b) * (f[3].r2 * f[2].r1 * f[1].r1);  // dz_ijk(3, 2, 1)
    const T v68 = (f[3].b * f[3].E * f[1].a) * (f[3].r3 * f[1].r1);  // dz_iji(3, 1)
    const T v69 = (f[3].a * f[3].E * f[1].b) * (f[3].r3 * f[1].r1);  // dz_iij(3, 1)
    const T v70 = (f[3].E * (f[2].s + f[2].b * f[2].a)) * (f[3].r2 * f[2].r2);  // dz_ijj(3, 2)
    const T v71 = (f[3].b * f[3].E * f[2].a) * (f[3].r3 * f[2].r1);  // dz_iji(3, 2)
    const T v72 = (f[3].a * f[3].E * f[2].b) * (f[3].r3 * f[2].r1);  // dz_iij(3, 2)
    const T v73 = f[3].DZs * f[3].r4;  // dz_iii(3,)
    const T v74 = f[0].PIs * f[0].r4;  // pi2_same(0,)
    const T v75 = T(0.5) * (f[1].pB * f[0].T1 + f[1].qB * f[0].T2) * (f[0].r3 * f[1].r1);  // pi2_triple(0, 1)
    const T v76 = T(0.5) * (f[2].pB * f[0].T1 + f[2].qB * f[0].T2) * (f[0].r3 * f[2].r1);  // pi2_triple(0, 2)
    const T v77 = T(0.5) * (f[3].pB * f[0].T1 + f[3].qB * f[0].T2) * (f[0].r3 * f[3].r1);  // pi2_triple(0, 3)
    const T v78 = (f[0].fA * f[1].fB) * (f[0].r2 * f[1].r2);  // pi2_iikk(0, 1)
    const T v79 = (f[1].fA * f[0].fB) * (f[1].r2 * f[0].r2);  // pi2_iikk(1, 0)
    const T v80 = T(0.5) * (f[0].fA * (f[1].pB * f[2].qB + f[1].qB * f[2].pB)) * (f[0].r2 * f[1].r1 * f[2].r1);  // pi2_iikl(0, 1, 2)
    const T v81 = T(0.5) * (f[0].fB * (f[1].pA * f[2].qA + f[1].qA * f[2].pA)) * (f[0].r2 * f[1].r1 * f[2].r1);  // pi2_ijkk(1, 2, 0)
    const T v82 = T(0.5) * (f[0].fA * (f[1].pB * f[3].qB + f[1].qB * f[3].pB)) * (f[0].r2 * f[1].r1 * f[3].r1);  // pi2_iikl(0, 1, 3)
    const T v83 = T(0.5) * (f[0].fB * (f[1].pA * f[3].qA + f[1].qA * f[3].pA)) * (f[0].r2 * f[1].r1 * f[3].r1);  // pi2_ijkk(1, 3, 0)
    const T v84 = (f[0].fA * f[2].fB) * (f[0].r2 * f[2].r2);  // pi2_iikk(0, 2)
    const T v85 = (f[2].fA * f[0].fB) * (f[2].r2 * f[0].r2);  // pi2_iikk(2, 0)
    const T v86 = T(0.5) * (f[0].fA * (f[2].pB * f[3].qB + f[2].qB * f[3].pB)) * (f[0].r2 * f[2].r1 * f[3].r1);  // pi2_iikl(0, 2, 3)
    const T v87 = T(0.5) * (f[0].fB * (f[2].pA * f[3].qA + f[2].qA * f[3].pA)) * (f[0].r2 * f[2].r1 * f[3].r1);  // pi2_ijkk(2, 3, 0)
    const T v88 = (f[0].fA * f[3].fB) * (f[0].r2 * f[3].r2);  // pi2_iikk(0, 3)
    const T v89 = (f[3].fA * f[0].fB) * (f[3].r2 * f[0].r2);  // pi2_iikk(3, 0)
    const T v90 = T(0.25) * ((f[0].pA * f[1].qA + f[0].qA * f[1].pA) * (f[0].pB * f[1].qB + f[0].qB * f[1].pB) + (f[0].Q1 * f[1].c4 + f[0].Q2 * f[1].c3 + f[0].Q3 * f[1].c2 + f[0].Q4 * f[1].c1 - (f[0].c1 * f[1].L1 + f[0].c2 * f[1].L2 + f[0].c3 * f[1].L3 + f[0].c4 * f[1].L4))) * (f[0].r2 * f[1].r2);  // pi2_ijij(0, 1)
    const T v91 = T(0.25) * ((f[1].pA * f[0].qA + f[1].qA * f[0].pA) * (f[1].pB * f[0].qB + f[1].qB * f[0].pB) + (f[1].Q1 * f[0].c4 + f[1].Q2 * f[0].c3 + f[1].Q3 * f[0].c2 + f[1].Q4 * f[0].c1 - (f[1].c1 * f[0].L1 + f[1].c2 * f[0].L2 + f[1].c3 * f[0].L3 + f[1].c4 * f[0].L4))) * (f[1].r2 * f[0].r2);  // pi2_ijij(1, 0)
    const T v92 = T(0.25) * (f[1].pA * (f[2].pB * (f[0].L1 - f[0].c4) + f[2].qB * (f[0].L2 - f[0].c3)) + f[1].qA * (f[2].pB * (f[0].L3 - f[0].c2) + f[2].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[1].r1 * f[2].r1);  // pi2_shared(0, 1, 2)
    const T v93 = T(0.25) * (f[2].pA * (f[1].pB * (f[0].L1 - f[0].c4) + f[1].qB * (f[0].L2 - f[0].c3)) + f[2].qA * (f[1].pB * (f[0].L3 - f[0].c2) + f[1].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[2].r1 * f[1].r1);  // pi2_shared(0, 2, 1)
    const T v94 = T(0.25) * (f[1].pA * (f[3].pB * (f[0].L1 - f[0].c4) + f[3].qB * (f[0].L2 - f[0].c3)) + f[1].qA * (f[3].pB * (f[0].L3 - f[0].c2) + f[3].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[1].r1 * f[3].r1);  // pi2_shared(0, 1, 3)
    const T v95 = T(0.25) * (f[3].pA * (f[1].pB * (f[0].L1 - f[0].c4) + f[1].qB * (f[0].L2 - f[0].c3)) + f[3].qA * (f[1].pB * (f[0].L3 - f[0].c2) + f[1].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[3].r1 * f[1].r1);  // pi2_shared(0, 3, 1)
    const T v96 = T(0.5) * (f[0].pB * f[1].T1 + f[0].qB * f[1].T2) * (f[1].r3 * f[0].r1);  // pi2_triple(1, 0)
    const T v97 = T(0.25) * (f[0].pA * (f[2].pB * (f[1].L1 - f[1].c4) + f[2].qB * (f[1].L2 - f[1].c3)) + f[0].qA * (f[2].pB * (f[1].L3 - f[1].c2) + f[2].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[0].r1 * f[2].r1);  // pi2_shared(1, 0, 2)
    const T v98 = T(0.25) * (f[2].pA * (f[0].pB * (f[1].L1 - f[1].c4) + f[0].qB * (f[1].L2 - f[1].c3)) + f[2].qA * (f[0].pB * (f[1].L3 - f[1].c2) + f[0].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[2].r1 * f[0].r1);  // pi2_shared(1, 2, 0)
    const T v99 = T(0.25) * (f[0].pA * (f[3].pB * (f[1].L1 - f[1].c4) + f[3].qB * (f[1].L2 - f[1].c3)) + f[0].qA * (f[3].pB * (f[1].L3 - f[1].c2) + f[3].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[0].r1 * f[3].r1);  // pi2_shared(1, 0, 3)
    const T v100 = T(0.25) * (f[3].pA * (f[0].pB * (f[1].L1 - f[1].c4) + f[0].qB * (f[1].L2 - f[1].c3)) + f[3].qA * (f[0].pB * (f[1].L3 - f[1].c2) + f[0].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[3].r1 * f[0].r1);  // pi2_shared(1, 3, 0)
    const T v101 = T(0.5) * (f[2].fB * (f[0].pA * f[1].qA + f[0].qA * f[1].pA)) * (f[2].r2 * f[0].r1 * f[1].r1);  // pi2_ijkk(0, 1, 2)
    const T v102 = T(0.5) * (f[2].fA * (f[0].pB * f[1].qB + f[0].qB * f[1].pB)) * (f[2].r2 * f[0].r1 * f[1].r1);  // pi2_iikl(2, 0, 1)
    const T v103 = T(0.25) * ((f[0].pA * f[1].qA + f[0].qA * f[1].pA) * (f[2].pB * f[3].qB + f[2].qB * f[3].pB)) * (f[0].r1 * f[1].r1 * f[2].r1 * f[3].r1);  // pi2_alldiff(0, 1, 2, 3)
    const T v104 = T(0.25) * ((f[2].pA * f[3].qA + f[2].qA * f[3].pA) * (f[0].pB * f[1].qB + f[0].qB * f[1].pB)) * (f[2].r1 * f[3].r1 * f[0].r1 * f[1].r1);  // pi2_alldiff(2, 3, 0, 1)
    const T v105 = T(0.5) * (f[3].fB * (f[0].pA * f[1].qA + f[0].qA * f[1].pA)) * (f[3].r2 * f[0].r1 * f[1].r1);  // pi2_ijkk(0, 1, 3)
    const T v106 = T(0.5) * (f[3].fA * (f[0].pB * f[1].qB + f[0].qB * f[1].pB)) * (f[3].r2 * f[0].r1 * f[1].r1);  // pi2_iikl(3, 0, 1)
    const T v107 = T(0.25) * ((f[0].pA * f[2].qA + f[0].qA * f[2].pA) * (f[0].pB * f[2].qB + f[0].qB * f[2].pB) + (f[0].Q1 * f[2].c4 + f[0].Q2 * f[2].c3 + f[0].Q3 * f[2].c2 + f[0].Q4 * f[2].c1 - (f[0].c1 * f[2].L1 + f[0].c2 * f[2].L2 + f[0].c3 * f[2].L3 + f[0].c4 * f[2].L4))) * (f[0].r2 * f[2].r2);  // pi2_ijij(0, 2)
    const T v108 = T(0.25) * ((f[2].pA * f[0].qA + f[2].qA * f[0].pA) * (f[2].pB * f[0].qB + f[2].qB * f[0].pB) + (f[2].Q1 * f[0].c4 + f[2].Q2 * f[0].c3 + f[2].Q3 * f[0].c2 + f[2].Q4 * f[0].c1 - (f[2].c1 * f[0].L1 + f[2].c2 * f[0].L2 + f[2].c3 * f[0].L3 + f[2].c4 * f[0].L4))) * (f[2].r2 * f[0].r2);  // pi2_ijij(2, 0)
    const T v109 = T(0.25) * (f[2].pA * (f[3].pB * (f[0].L1 - f[0].c4) + f[3].qB * (f[0].L2 - f[0].c3)) + f[2].qA * (f[3].pB * (f[0].L3 - f[0].c2) + f[3].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[2].r1 * f[3].r1);  // pi2_shared(0, 2, 3)
    const T v110 = T(0.25) * (f[3].pA * (f[2].pB * (f[0].L1 - f[0].c4) + f[2].qB * (f[0].L2 - f[0].c3)) + f[3].qA * (f[2].pB * (f[0].L3 - f[0].c2) + f[2].qB * (f[0].L4 - f[0].c1))) * (f[0].r2 * f[3].r1 * f[2].r1);  // pi2_shared(0, 3, 2)
    const T v111 = T(0.5) * (f[1].fB * (f[0].pA * f[2].qA + f[0].qA * f[2].pA)) * (f[1].r2 * f[0].r1 * f[2].r1);  // pi2_ijkk(0, 2, 1)
    const T v112 = T(0.5) * (f[1].fA * (f[0].pB * f[2].qB + f[0].qB * f[2].pB)) * (f[1].r2 * f[0].r1 * f[2].r1);  // pi2_iikl(1, 0, 2)
    const T v113 = T(0.25) * (f[0].pA * (f[1].pB * (f[2].L1 - f[2].c4) + f[1].qB * (f[2].L2 - f[2].c3)) + f[0].qA * (f[1].pB * (f[2].L3 - f[2].c2) + f[1].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[0].r1 * f[1].r1);  // pi2_shared(2, 0, 1)
    const T v114 = T(0.25) * (f[1].pA * (f[0].pB * (f[2].L1 - f[2].c4) + f[0].qB * (f[2].L2 - f[2].c3)) + f[1].qA * (f[0].pB * (f[2].L3 - f[2].c2) + f[0].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[1].r1 * f[0].r1);  // pi2_shared(2, 1, 0)
    const T v115 = T(0.25) * ((f[0].pA * f[2].qA + f[0].qA * f[2].pA) * (f[1].pB * f[3].qB + f[1].qB * f[3].pB)) * (f[0].r1 * f[2].r1 * f[1].r1 * f[3].r1);  // pi2_alldiff(0, 2, 1, 3)
    const T v116 = T(0.25) * ((f[1].pA * f[3].qA + f[1].qA * f[3].pA) * (f[0].pB * f[2].qB + f[0].qB * f[2].pB)) * (f[1].r1 * f[3].r1 * f[0].r1 * f[2].r1);  // pi2_alldiff(1, 3, 0, 2)
    const T v117 = T(0.5) * (f[0].pB * f[2].T1 + f[0].qB * f[2].T2) * (f[2].r3 * f[0].r1);  // pi2_triple(2, 0)
    const T v118 = T(0.25) * (f[0].pA * (f[3].pB * (f[2].L1 - f[2].c4) + f[3].qB * (f[2].L2 - f[2].c3)) + f[0].qA * (f[3].pB * (f[2].L3 - f[2].c2) + f[3].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[0].r1 * f[3].r1);  // pi2_shared(2, 0, 3)
    const T v119 = T(0.25) * (f[3].pA * (f[0].pB * (f[2].L1 - f[2].c4) + f[0].qB * (f[2].L2 - f[2].c3)) + f[3].qA * (f[0].pB * (f[2].L3 - f[2].c2) + f[0].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[3].r1 * f[0].r1);  // pi2_shared(2, 3, 0)
    const T v120 = T(0.5) * (f[3].fB * (f[0].pA * f[2].qA + f[0].qA * f[2].pA)) * (f[3].r2 * f[0].r1 * f[2].r1);  // pi2_ijkk(0, 2, 3)
    const T v121 = T(0.5) * (f[3].fA * (f[0].pB * f[2].qB + f[0].qB * f[2].pB)) * (f[3].r2 * f[0].r1 * f[2].r1);  // pi2_iikl(3, 0, 2)
    const T v122 = T(0.25) * ((f[0].pA * f[3].qA + f[0].qA * f[3].pA) * (f[0].pB * f[3].qB + f[0].qB * f[3].pB) + (f[0].Q1 * f[3].c4 + f[0].Q2 * f[3].c3 + f[0].Q3 * f[3].c2 + f[0].Q4 * f[3].c1 - (f[0].c1 * f[3].L1 + f[0].c2 * f[3].L2 + f[0].c3 * f[3].L3 + f[0].c4 * f[3].L4))) * (f[0].r2 * f[3].r2);  // pi2_ijij(0, 3)
    const T v123 = T(0.25) * ((f[3].pA * f[0].qA + f[3].qA * f[0].pA) * (f[3].pB * f[0].qB + f[3].qB * f[0].pB) + (f[3].Q1 * f[0].c4 + f[3].Q2 * f[0].c3 + f[3].Q3 * f[0].c2 + f[3].Q4 * f[0].c1 - (f[3].c1 * f[0].L1 + f[3].c2 * f[0].L2 + f[3].c3 * f[0].L3 + f[3].c4 * f[0].L4))) * (f[3].r2 * f[0].r2);  // pi2_ijij(3, 0)
    const T v124 = T(0.5) * (f[1].fB * (f[0].pA * f[3].qA + f[0].qA * f[3].pA)) * (f[1].r2 * f[0].r1 * f[3].r1);  // pi2_ijkk(0, 3, 1)
    const T v125 = T(0.5) * (f[1].fA * (f[0].pB * f[3].qB + f[0].qB * f[3].pB)) * (f[1].r2 * f[0].r1 * f[3].r1);  // pi2_iikl(1, 0, 3)
    const T v126 = T(0.25) * ((f[0].pA * f[3].qA + f[0].qA * f[3].pA) * (f[1].pB * f[2].qB + f[1].qB * f[2].pB)) * (f[0].r1 * f[3].r1 * f[1].r1 * f[2].r1);  // pi2_alldiff(0, 3, 1, 2)
    const T v127 = T(0.25) * ((f[1].pA * f[2].qA + f[1].qA * f[2].pA) * (f[0].pB * f[3].qB + f[0].qB * f[3].pB)) * (f[1].r1 * f[2].r1 * f[0].r1 * f[3].r1);  // pi2_alldiff(1, 2, 0, 3)
    const T v128 = T(0.25) * (f[0].pA * (f[1].pB * (f[3].L1 - f[3].c4) + f[1].qB * (f[3].L2 - f[3].c3)) + f[0].qA * (f[1].pB * (f[3].L3 - f[3].c2) + f[1].qB * (f[3].L4 - f[3].c1))) * (f[3].r2 * f[0].r1 * f[1].r1);  // pi2_shared(3, 0, 1)
    const T v129 = T(0.25) * (f[1].pA * (f[0].pB * (f[3].L1 - f[3].c4) + f[0].qB * (f[3].L2 - f[3].c3)) + f[1].qA * (f[0].pB * (f[3].L3 - f[3].c2) + f[0].qB * (f[3].L4 - f[3].c1))) * (f[3].r2 * f[1].r1 * f[0].r1);  // pi2_shared(3, 1, 0)
    const T v130 = T(0.5) * (f[2].fB * (f[0].pA * f[3].qA + f[0].qA * f[3].pA)) * (f[2].r2 * f[0].r1 * f[3].r1);  // pi2_ijkk(0, 3, 2)
    const T v131 = T(0.5) * (f[2].fA * (f[0].pB * f[3].qB + f[0].qB * f[3].pB)) * (f[2].r2 * f[0].r1 * f[3].r1);  // pi2_iikl(2, 0, 3)
    const T v132 = T(0.25) * (f[0].pA * (f[2].pB * (f[3].L1 - f[3].c4) + f[2].qB * (f[3].L2 - f[3].c3)) + f[0].qA * (f[2].pB * (f[3].L3 - f[3].c2) + f[2].qB * (f[3].L4 - f[3].c1))) * (f[3].r2 * f[0].r1 * f[2].r1);  // pi2_shared(3, 0, 2)
    const T v133 = T(0.25) * (f[2].pA * (f[0].pB * (f[3].L1 - f[3].c4) + f[0].qB * (f[3].L2 - f[3].c3)) + f[2].qA * (f[0].pB * (f[3].L3 - f[3].c2) + f[0].qB * (f[3].L4 - f[3].c1))) * (f[3].r2 * f[2].r1 * f[0].r1);  // pi2_shared(3, 2, 0)
    const T v134 = T(0.5) * (f[0].pB * f[3].T1 + f[0].qB * f[3].T2) * (f[3].r3 * f[0].r1);  // pi2_triple(3, 0)
    const T v135 = f[1].PIs * f[1].r4;  // pi2_same(1,)
    const T v136 = T(0.5) * (f[2].pB * f[1].T1 + f[2].qB * f[1].T2) * (f[1].r3 * f[2].r1);  // pi2_triple(1, 2)
    const T v137 = T(0.5) * (f[3].pB * f[1].T1 + f[3].qB * f[1].T2) * (f[1].r3 * f[3].r1);  // pi2_triple(1, 3)
    const T v138 = (f[1].fA * f[2].fB) * (f[1].r2 * f[2].r2);  // pi2_iikk(1, 2)
    const T v139 = (f[2].fA * f[1].fB) * (f[2].r2 * f[1].r2);  // pi2_iikk(2, 1)
    const T v140 = T(0.5) * (f[1].fA * (f[2].pB * f[3].qB + f[2].qB * f[3].pB)) * (f[1].r2 * f[2].r1 * f[3].r1);  // pi2_iikl(1, 2, 3)
    const T v141 = T(0.5) * (f[1].fB * (f[2].pA * f[3].qA + f[2].qA * f[3].pA)) * (f[1].r2 * f[2].r1 * f[3].r1);  // pi2_ijkk(2, 3, 1)
    const T v142 = (f[1].fA * f[3].fB) * (f[1].r2 * f[3].r2);  // pi2_iikk(1, 3)
    const T v143 = (f[3].fA * f[1].fB) * (f[3].r2 * f[1].r2);  // pi2_iikk(3, 1)
    const T v144 = T(0.25) * ((f[1].pA * f[2].qA + f[1].qA * f[2].pA) * (f[1].pB * f[2].qB + f[1].qB * f[2].pB) + (f[1].Q1 * f[2].c4 + f[1].Q2 * f[2].c3 + f[1].Q3 * f[2].c2 + f[1].Q4 * f[2].c1 - (f[1].c1 * f[2].L1 + f[1].c2 * f[2].L2 + f[1].c3 * f[2].L3 + f[1].c4 * f[2].L4))) * (f[1].r2 * f[2].r2);  // pi2_ijij(1, 2)
    const T v145 = T(0.25) * ((f[2].pA * f[1].qA + f[2].qA * f[1].pA) * (f[2].pB * f[1].qB + f[2].qB * f[1].pB) + (f[2].Q1 * f[1].c4 + f[2].Q2 * f[1].c3 + f[2].Q3 * f[1].c2 + f[2].Q4 * f[1].c1 - (f[2].c1 * f[1].L1 + f[2].c2 * f[1].L2 + f[2].c3 * f[1].L3 + f[2].c4 * f[1].L4))) * (f[2].r2 * f[1].r2);  // pi2_ijij(2, 1)
    const T v146 = T(0.25) * (f[2].pA * (f[3].pB * (f[1].L1 - f[1].c4) + f[3].qB * (f[1].L2 - f[1].c3)) + f[2].qA * (f[3].pB * (f[1].L3 - f[1].c2) + f[3].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[2].r1 * f[3].r1);  // pi2_shared(1, 2, 3)
    const T v147 = T(0.25) * (f[3].pA * (f[2].pB * (f[1].L1 - f[1].c4) + f[2].qB * (f[1].L2 - f[1].c3)) + f[3].qA * (f[2].pB * (f[1].L3 - f[1].c2) + f[2].qB * (f[1].L4 - f[1].c1))) * (f[1].r2 * f[3].r1 * f[2].r1);  // pi2_shared(1, 3, 2)
    const T v148 = T(0.5) * (f[1].pB * f[2].T1 + f[1].qB * f[2].T2) * (f[2].r3 * f[1].r1);  // pi2_triple(2, 1)
    const T v149 = T(0.25) * (f[1].pA * (f[3].pB * (f[2].L1 - f[2].c4) + f[3].qB * (f[2].L2 - f[2].c3)) + f[1].qA * (f[3].pB * (f[2].L3 - f[2].c2) + f[3].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[1].r1 * f[3].r1);  // pi2_shared(2, 1, 3)
    const T v150 = T(0.25) * (f[3].pA * (f[1].pB * (f[2].L1 - f[2].c4) + f[1].qB * (f[2].L2 - f[2].c3)) + f[3].qA * (f[1].pB * (f[2].L3 - f[2].c2) + f[1].qB * (f[2].L4 - f[2].c1))) * (f[2].r2 * f[3].r1 * f[1].r1);  // pi2_shared(2, 3, 1)
    const T v151 = T(0.5) * (f[3].fB * (f[1].pA * f[2].qA + f[1].qA * f[2].pA)) * (f[3].r2 * f[1].r1 * f[2].r1);  // pi2_ijkk(1, 2, 3)
    const T v152 = T(0.5) * (f[3].fA * (f[1].pB * f[2].qB + f[1].qB * f[2].pB)) * (f[3].r2 * f[1].r1 * f[2].r1);  // pi2_iikl(3, 1, 2)
    const T v153 = T(0.25) * ((f[1].pA * f[3].qA + f[1].qA * f[3].pA) * (f[1].pB * f[3].qB + f[1].qB * f[3].pB) + (f[1].Q1 * f[3].c4 + f[1].Q2 * f[3].c3 + f[1].Q3 * f[3].c2 + f[1].Q4 * f[3].c1 - (f[1].c1 * f[3].L1 + f[1].c2 * f[3].L2 + f[1].c3 * f[3].L3 + f[1].c4 * f[3].L4))) * (f[1].r2 * f[3].r2);  // pi2_ijij(1, 3)
    const T v154 = T(0.25) * ((f[3].pA * f[1].qA + f[3].qA * f[1].pA) * (f[3].pB * f[1].qB + f[3].qB * f[1].pB) + (f[3].Q1 * f[1].c4 + f[3].Q2 * f[1].c3 + f[3].Q3 * f[1].c2 + f[3].Q4 * f[1].c1 - (f[3].c1 * f[1].L1 + f[3].c2 * f[1].L2 + f[3].c3 * f[1].L3 + f[3].c4 * f[1].L4))) * (f[3].r2 * f[1].r2);  // pi2_ijij(3, 1)
    const T v155 = T(0.5) * (f[2].fB * (f[1].pA * f[3].qA + f[1].qA * f[3].pA)) * (f[2].r2 * f[1].r1 * f[3].r1);  // pi2_ijkk(1, 3, 2)
    const T v156 = T(0.5) * (f[2].fA * (f[1].pB * f[3].qB + f[1].qB * f[3].pB)) * (f[2].r2 * f[1].r1 * f[3].r1);  // pi2_iikl(2, 1, 3)
    const T v157 = T(0.25) * (f[1].pA * (f[2].pB * (f[3].L1 - f[3].c4) + f[2].qB * (f[3].L2 - f[3].c3)) + f[1].qA * (f[2].pB * (f[3].L3 - f[3].c2) + f[2].qB * (f[3].L4 - f[3].c1))) * (f[3].r2 * f[1].r1 * f[2].r1);  // pi2_shared(3, 1, 2)
    const T v158 = T(0.25) * (f[2].pA * (f[1].pB * (f[3].L1 - f[3].c4) + f[1].qB * (f[3].L2 - f[3].c3)) + f[2].qA * (f[1].pB * (f[3].L3 - f[3].c2) + f[1].qB * (f[3].L4 - f[3].c1))) * (f[3].r2 * f[2].r1 * f[1].r1);  // pi2_shared(3, 2, 1)
    const T v159 = T(0.5) * (f[1].pB * f[3].T1 + f[1].qB * f[3].T2) * (f[3].r3 * f[1].r1);  // pi2_triple(3, 1)
    const T v160 = f[2].PIs * f[2].r4;  // pi2_same(2,)
    const T v161 = T(0.5) * (f[3].pB * f[2].T1 + f[3].qB * f[2].T2) * (f[2].r3 * f[3].r1);  // pi2_triple(2, 3)
    const T v162 = (f[2].fA * f[3].fB) * (f[2].r2 * f[3].r2);  // pi2_iikk(2, 3)
    const T v163 = (f[3].fA * f[2].fB) * (f[3].r2 * f[2].r2);  // pi2_iikk(3, 2)
    const T v164 = T(0.25) * ((f[2].pA * f[3].qA + f[2].qA * f[3].pA) * (f[2].pB * f[3].qB + f[2].qB * f[3].pB) + (f[2].Q1 * f[3].c4 + f[2].Q2 * f[3].c3 + f[2].Q3 * f[3].c2 + f[2].Q4 * f[3].c1 - (f[2].c1 * f[3].L1 + f[2].c2 * f[3].L2 + f[2].c3 * f[3].L3 + f[2].c4 * f[3].L4))) * (f[2].r2 * f[3].r2);  // pi2_ijij(2, 3)
    const T v165 = T(0.25) * ((f[3].pA * f[2].qA + f[3].qA * f[2].pA) * (f[3].pB * f[2].qB + f[3].qB * f[2].pB) + (f[3].Q1 * f[2].c4 + f[3].Q2 * f[2].c3 + f[3].Q3 * f[2].c2 + f[3].Q4 * f[2].c1 - (f[3].c1 * f[2].L1 + f[3].c2 * f[2].L2 + f[3].c3 * f[2].L3 + f[3].c4 * f[2].L4))) * (f[3].r2 * f[2].r2);  // pi2_ijij(3, 2)
    const T v166 = T(0.5) * (f[2].pB * f[3].T1 + f[2].qB * f[3].T2) * (f[3].r3 * f[2].r1);  // pi2_triple(3, 2)
    const T v167 = f[3].PIs * f[3].r4;  // pi2_same(3,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // DD_0_1
    acc[2] += v2;  // DD_0_2
    acc[3] += v3;  // DD_0_3
    acc[4] += v4;  // DD_1_1
    acc[5] += v5;  // DD_1_2
    acc[6] += v6;  // DD_1_3
    acc[7] += v7;  // DD_2_2
    acc[8] += v8;  // DD_2_3
    acc[9] += v9;  // DD_3_3
    acc[10] += v10;  // Dz_0_0_0
    acc[11] += T(0.5) * (v11 + v12);  // Dz_0_0_1
    acc[12] += T(0.5) * (v13 + v14);  // Dz_0_0_2
    acc[13] += T(0.5) * (v15 + v16);  // Dz_0_0_3
    acc[14] += v17;  // Dz_0_1_1
    acc[15] += T(0.5) * (v18 + v19);  // Dz_0_1_2
    acc[16] += T(0.5) * (v20 + v21);  // Dz_0_1_3
    acc[17] += v22;  // Dz_0_2_2
    acc[18] += T(0.5) * (v23 + v24);  // Dz_0_2_3
    acc[19] += v25;  // Dz_0_3_3
    acc[20] += v26;  // Dz_1_0_0
    acc[21] += T(0.5) * (v27 + v28);  // Dz_1_0_1
    acc[22] += T(0.5) * (v29 + v30);  // Dz_1_0_2
    acc[23] += T(0.5) * (v31 + v32);  // Dz_1_0_3
    acc[24] += v33;  // Dz_1_1_1
    acc[25] += T(0.5) * (v34 + v35);  // Dz_1_1_2
    acc[26] += T(0.5) * (v36 + v37);  // Dz_1_1_3
    acc[27] += v38;  // Dz_1_2_2
    acc[28] += T(0.5) * (v39 + v40);  // Dz_1_2_3
    acc[29] += v41;  // Dz_1_3_3
    acc[30] += v42;  // Dz_2_0_0
    acc[31] += T(0.5) * (v43 + v44);  // Dz_2_0_1
    acc[32] += T(0.5) * (v45 + v46);  // Dz_2_0_2
    acc[33] += T(0.5) * (v47 + v48);  // Dz_2_0_3
    acc[34] += v49;  // Dz_2_1_1
    acc[35] += T(0.5) * (v50 + v51);  // Dz_2_1_2
    acc[36] += T(0.5) * (v52 + v53);  // Dz_2_1_3
    acc[37] += v54;  // Dz_2_2_2
    acc[38] += T(0.5) * (v55 + v56);  // Dz_2_2_3
    acc[39] += v57;  // Dz_2_3_3
    acc[40] += v58;  // Dz_3_0_0
    acc[41] += T(0.5) * (v59 + v60);  // Dz_3_0_1
    acc[42] += T(0.5) * (v61 + v62);  // Dz_3_0_2
    acc[43] += T(0.5) * (v63 + v64);  // Dz_3_0_3
    acc[44] += v65;  // Dz_3_1_1
    acc[45] += T(0.5) * (v66 + v67);  // Dz_3_1_2
    acc[46] += T(0.5) * (v68 + v69);  // Dz_3_1_3
    acc[47] += v70;  // Dz_3_2_2
    acc[48] += T(0.5) * (v71 + v72);  // Dz_3_2_3
    acc[49] += v73;  // Dz_3_3_3
    acc[50] += v74;  // pi2_0_0_0_0
    acc[51] += v75;  // pi2_0_0_0_1
    acc[52] += v76;  // pi2_0_0_0_2
    acc[53] += v77;  // pi2_0_0_0_3
    acc[54] += T(0.5) * (v78 + v79);  // pi2_0_0_1_1
    acc[55] += T(0.5) * (v80 + v81);  // pi2_0_0_1_2
    acc[56] += T(0.5) * (v82 + v83);  // pi2_0_0_1_3
    acc[57] += T(0.5) * (v84 + v85);  // pi2_0_0_2_2
    acc[58] += T(0.5) * (v86 + v87);  // pi2_0_0_2_3
    acc[59] += T(0.5) * (v88 + v89);  // pi2_0_0_3_3
    acc[60] += T(0.5) * (v90 + v91);  // pi2_0_1_0_1
    acc[61] += T(0.5) * (v92 + v93);  // pi2_0_1_0_2
    acc[62] += T(0.5) * (v94 + v95);  // pi2_0_1_0_3
    acc[63] += v96;  // pi2_0_1_1_1
    acc[64] += T(0.5) * (v97 + v98);  // pi2_0_1_1_2
    acc[65] += T(0.5) * (v99 + v100);  // pi2_0_1_1_3
    acc[66] += T(0.5) * (v101 + v102);  // pi2_0_1_2_2
    acc[67] += T(0.5) * (v103 + v104);  // pi2_0_1_2_3
    acc[68] += T(0.5) * (v105 + v106);  // pi2_0_1_3_3
    acc[69] += T(0.5) * (v107 + v108);  // pi2_0_2_0_2
    acc[70] += T(0.5) * (v109 + v110);  // pi2_0_2_0_3
    acc[71] += T(0.5) * (v111 + v112);  // pi2_0_2_1_1
    acc[72] += T(0.5) * (v113 + v114);  // pi2_0_2_1_2
    acc[73] += T(0.5) * (v115 + v116);  // pi2_0_2_1_3
    acc[74] += v117;  // pi2_0_2_2_2
    acc[75] += T(0.5) * (v118 + v119);  // pi2_0_2_2_3
    acc[76] += T(0.5) * (v120 + v121);  // pi2_0_2_3_3
    acc[77] += T(0.5) * (v122 + v123);  // pi2_0_3_0_3
    acc[78] += T(0.5) * (v124 + v125);  // pi2_0_3_1_1
    acc[79] += T(0.5) * (v126 + v127);  // pi2_0_3_1_2
    acc[80] += T(0.5) * (v128 + v129);  // pi2_0_3_1_3
    acc[81] += T(0.5) * (v130 + v131);  // pi2_0_3_2_2
    acc[82] += T(0.5) * (v132 + v133);  // pi2_0_3_2_3
    acc[83] += v134;  // pi2_0_3_3_3
    acc[84] += v135;  // pi2_1_1_1_1
    acc[85] += v136;  // pi2_1_1_1_2
    acc[86] += v137;  // pi2_1_1_1_3
    acc[87] += T(0.5) * (v138 + v139);  // pi2_1_1_2_2
    acc[88] += T(0.5) * (v140 + v141);  // pi2_1_1_2_3
    acc[89] += T(0.5) * (v142 + v143);  // pi2_1_1_3_3
    acc[90] += T(0.5) * (v144 + v145);  // pi2_1_2_1_2
    acc[91] += T(0.5) * (v146 + v147);  // pi2_1_2_1_3
    acc[92] += v148;  // pi2_1_2_2_2
    acc[93] += T(0.5) * (v149 + v150);  // pi2_1_2_2_3
    acc[94] += T(0.5) * (v151 + v152);  // pi2_1_2_3_3
    acc[95] += T(0.5) * (v153 + v154);  // pi2_1_3_1_3
    acc[96] += T(0.5) * (v155 + v156);  // pi2_1_3_2_2
    acc[97] += T(0.5) * (v157 + v158);  // pi2_1_3_2_3
    acc[98] += v159;  // pi2_1_3_3_3
    acc[99] += v160;  // pi2_2_2_2_2
    acc[100] += v161;  // pi2_2_2_2_3
    acc[101] += T(0.5) * (v162 + v163);  // pi2_2_2_3_3
    acc[102] += T(0.5) * (v164 + v165);  // pi2_2_3_2_3
    acc[103] += v166;  // pi2_2_3_3_3
    acc[104] += v167;  // pi2_3_3_3_3
}

#include "ldk_geno_feat.cuh"
// genotype path, P = 1: 3 statistics from 3 distinct raw calls
template <typename T>
LDK_DEV void geno_features_P1(GenoFeat<T>& x) {
    geno_prepare(x);
    x.xAB = x.g1 + T(0.5) * x.g2 + T(0.5) * x.g4 + T(0.25) * x.g5;
    x.xAb = T(0.5) * x.g2 + x.g3 + T(0.25) * x.g5 + T(0.5) * x.g6;
    x.xaB = T(0.5) * x.g4 + T(0.25) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.xab = T(0.25) * x.g5 + T(0.5) * x.g6 + T(0.5) * x.g8 + x.g9;
    x.D = x.xAB * x.xab - x.xAb * x.xaB;
    x.pA = x.g1 + x.g2 + x.g3 + T(0.5) * (x.g4 + x.g5 + x.g6);
    x.qA = T(0.5) * (x.g4 + x.g5 + x.g6) + x.g7 + x.g8 + x.g9;
    x.pB = x.g1 + T(0.5) * x.g2 + x.g4 + T(0.5) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.qB = T(0.5) * x.g2 + x.g3 + T(0.5) * x.g5 + x.g6 + T(0.5) * x.g8 + x.g9;
    x.p = x.pA * x.invn;
    x.q = x.pB * x.invn;
    x.A = -x.g1 + x.g3 - x.g4 + x.g6 - x.g7 + x.g9;
    x.Bv = -x.g1 - x.g2 - x.g3 + x.g7 + x.g8 + x.g9;
    x.DD1 = T(4) * (((x.g2 * x.g4 - x.g2 * x.g2 * x.g4 + T(4) * x.g3 * x.g4 - T(4) * x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4) + (-x.g2 * x.g4 * x.g4 - T(4) * x.g3 * x.g4 * x.g4) + (x.g1 * x.g5 - x.g1 * x.g1 * x.g5 + x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g3 * x.g3 * x.g5 - T(4) * x.g3 * x.g4 * x.g5 - x.g1 * x.g5 * x.g5 - x.g3 * x.g5 * x.g5) + (T(4) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 + x.g2 * x.g6 - T(4) * x.g1 * x.g2 * x.g6 - x.g2 * x.g2 * x.g6 + T(2) * x.g2 * x.g4 * x.g6 - T(4) * x.g1 * x.g5 * x.g6 - T(4) * x.g1 * x.g6 * x.g6 - x.g2 * x.g6 * x.g6) + (T(4) * x.g2 * x.g7 - T(4) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7 - T(16) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(4) * x.g2 * x.g4 * x.g7 - T(16) * x.g3 * x.g4 * x.g7 + x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 - T(4) * x.g2 * x.g5 * x.g7 - T(18) * x.g3 * x.g5 * x.g7 - x.g5 * x.g5 * x.g7 + T(4) * x.g6 * x.g7 + T(8) * x.g1 * x.g6 * x.g7 - T(16) * x.g3 * x.g6 * x.g7 - T(4) * x.g5 * x.g6 * x.g7 - T(4) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7) + (T(4) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 + T(4) * x.g3 * x.g8 + T(8) * x.g1 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 + x.g4 * x.g8 - T(4) * x.g1 * x.g4 * x.g8 + T(2) * x.g2 * x.g4 * x.g8 - x.g4 * x.g4 * x.g8 - T(4) * x.g1 * x.g5 * x.g8 - T(4) * x.g3 * x.g5 * x.g8 + x.g6 * x.g8 + T(2) * x.g2 * x.g6 * x.g8 - T(4) * x.g3 * x.g6 * x.g8 + T(2) * x.g4 * x.g6 * x.g8 - x.g6 * x.g6 * x.g8 - T(16) * x.g3 * x.g7 * x.g8 - T(4) * x.g6 * x.g7 * x.g8 - T(4) * x.g1 * x.g8 * x.g8 - T(4) * x.g3 * x.g8 * x.g8 - x.g4 * x.g8 * x.g8 - x.g6 * x.g8 * x.g8) + (T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9 + T(4) * x.g2 * x.g9 - T(16) * x.g1 * x.g2 * x.g9 - T(4) * x.g2 * x.g2 * x.g9 + T(4) * x.g4 * x.g9 - T(16) * x.g1 * x.g4 * x.g9 + T(8) * x.g3 * x.g4 * x.g9 - T(4) * x.g4 * x.g4 * x.g9 + x.g5 * x.g9 - T(18) * x.g1 * x.g5 * x.g9 - T(4) * x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 - T(4) * x.g4 * x.g5 * x.g9 - x.g5 * x.g5 * x.g9 - T(16) * x.g1 * x.g6 * x.g9 - T(4) * x.g2 * x.g6 * x.g9 + T(8) * x.g2 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 - T(16) * x.g1 * x.g8 * x.g9 - T(4) * x.g4 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - x.g5 * x.g9 * x.g9) ) * T(0.0625) + x.D * x.D) * x.w4;
    x.DZ1 = T(2) * (T(0.25) * (-(x.g2 * x.g4) + T(3) * x.g1 * x.g2 * x.g4 + x.g2 * x.g2 * x.g4 + T(2) * x.g3 * x.g4 + T(4) * x.g1 * x.g3 * x.g4 - x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4 + x.g2 * x.g4 * x.g4 + T(2) * x.g3 * x.g4 * x.g4 + T(2) * x.g1 * x.g5 - T(3) * x.g1 * x.g1 * x.g5 - x.g1 * x.g2 * x.g5 + T(2) * x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g2 * x.g3 * x.g5 - T(3) * x.g3 * x.g3 * x.g5 - x.g1 * x.g4 * x.g5 + x.g3 * x.g4 * x.g5 + T(2) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 - x.g2 * x.g6 - x.g1 * x.g2 * x.g6 + x.g2 * x.g2 * x.g6 + T(4) * x.g1 * x.g3 * x.g6 + T(3) * x.g2 * x.g3 * x.g6 - T(2) * x.g1 * x.g4 * x.g6 - T(2) * x.g2 * x.g4 * x.g6 - T(2) * x.g3 * x.g4 * x.g6 + x.g1 * x.g5 * x.g6 - x.g3 * x.g5 * x.g6 + T(2) * x.g1 * x.g6 * x.g6 + x.g2 * x.g6 * x.g6 + T(2) * x.g2 * x.g7 + T(4) * x.g1 * x.g2 * x.g7 + T(2) * x.g2 * x.g2 * x.g7 + T(8) * x.g3 * x.g7 + T(4) * x.g1 * x.g3 * x.g7 - T(4) * x.g3 * x.g3 * x.g7 - x.g2 * x.g4 * x.g7 + T(2) * x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 + x.g2 * x.g5 * x.g7 + T(2) * x.g3 * x.g5 * x.g7 - x.g4 * x.g5 * x.g7 + T(2) * x.g6 * x.g7 - x.g2 * x.g6 * x.g7 - T(2) * x.g4 * x.g6 * x.g7 + x.g5 * x.g6 * x.g7 + T(2) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(4) * x.g3 * x.g7 * x.g7 - T(3) * x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7 + T(2) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 - T(2) * x.g1 * x.g2 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g2 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 - x.g4 * x.g8 - x.g1 * x.g4 * x.g8 - T(2) * x.g2 * x.g4 * x.g8 - x.g3 * x.g4 * x.g8 + x.g4 * x.g4 * x.g8 + x.g1 * x.g5 * x.g8 + x.g3 * x.g5 * x.g8 - x.g6 * x.g8 - x.g1 * x.g6 * x.g8 - T(2) * x.g2 * x.g6 * x.g8 - x.g3 * x.g6 * x.g8 - T(2) * x.g4 * x.g6 * x.g8 + x.g6 * x.g6 * x.g8 + T(4) * x.g1 * x.g7 * x.g8 - T(2) * x.g2 * x.g7 * x.g8 + T(3) * x.g4 * x.g7 * x.g8 - x.g5 * x.g7 * x.g8 - x.g6 * x.g7 * x.g8 + T(2) * x.g1 * x.g8 * x.g8 + T(2) * x.g3 * x.g8 * x.g8 + x.g4 * x.g8 * x.g8 + x.g6 * x.g8 * x.g8 + T(8) * x.g1 * x.g9 - T(4) * x.g1 * x.g1 * x.g9 + T(2) * x.g2 * x.g9 + T(2) * x.g2 * x.g2 * x.g9 + T(4) * x.g1 * x.g3 * x.g9 + T(4) * x.g2 * x.g3 * x.g9 + T(2) * x.g4 * x.g9 - x.g2 * x.g4 * x.g9 + T(2) * x.g4 * x.g4 * x.g9 + T(2) * x.g5 * x.g9 + T(2) * x.g1 * x.g5 * x.g9 + x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 + x.g4 * x.g5 * x.g9 - x.g2 * x.g6 * x.g9 - T(2) * x.g4 * x.g6 * x.g9 - x.g5 * x.g6 * x.g9 + T(4) * x.g1 * x.g7 * x.g9 + T(4) * x.g3 * x.g7 * x.g9 + T(4) * x.g4 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 + T(4) * x.g6 * x.g7 * x.g9 - T(2) * x.g2 * x.g8 * x.g9 + T(4) * x.g3 * x.g8 * x.g9 - x.g4 * x.g8 * x.g9 - x.g5 * x.g8 * x.g9 + T(3) * x.g6 * x.g8 * x.g9 - T(4) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - T(3) * x.g5 * x.g9 * x.g9 ) + x.A * x.Bv * x.D) * x.w4;
    x.PI1 = (x.pA * x.pB * x.qB * x.qA + ((T(13) * x.g2 * x.g4 - T(16) * x.g1 * x.g2 * x.g4 - T(11) * x.g2 * x.g2 * x.g4 + T(16) * x.g3 * x.g4 - T(28) * x.g1 * x.g3 * x.g4 - T(24) * x.g2 * x.g3 * x.g4) + (-T(8) * x.g3 * x.g3 * x.g4 - T(11) * x.g2 * x.g4 * x.g4 - T(20) * x.g3 * x.g4 * x.g4 - T(6) * x.g5 + T(12) * x.g1 * x.g5 - T(4) * x.g1 * x.g1 * x.g5 + T(17) * x.g2 * x.g5) + (-T(20) * x.g1 * x.g2 * x.g5 - T(11) * x.g2 * x.g2 * x.g5 + T(12) * x.g3 * x.g5 - T(28) * x.g1 * x.g3 * x.g5 - T(20) * x.g2 * x.g3 * x.g5 - T(4) * x.g3 * x.g3 * x.g5) + (T(17) * x.g4 * x.g5 - T(20) * x.g1 * x.g4 * x.g5 - T(32) * x.g2 * x.g4 * x.g5 - T(40) * x.g3 * x.g4 * x.g5 - T(11) * x.g4 * x.g4 * x.g5 + T(11) * x.g5 * x.g5) + (-T(16) * x.g1 * x.g5 * x.g5 - T(17) * x.g2 * x.g5 * x.g5 - T(16) * x.g3 * x.g5 * x.g5 - T(17) * x.g4 * x.g5 * x.g5 - T(6) * x.g5 * x.g5 * x.g5 + T(16) * x.g1 * x.g6 - T(8) * x.g1 * x.g1 * x.g6) + (T(13) * x.g2 * x.g6 - T(24) * x.g1 * x.g2 * x.g6 - T(11) * x.g2 * x.g2 * x.g6 - T(28) * x.g1 * x.g3 * x.g6 - T(16) * x.g2 * x.g3 * x.g6 + T(24) * x.g4 * x.g6) + (-T(36) * x.g1 * x.g4 * x.g6 - T(38) * x.g2 * x.g4 * x.g6 - T(36) * x.g3 * x.g4 * x.g6 - T(20) * x.g4 * x.g4 * x.g6 + T(17) * x.g5 * x.g6 - T(40) * x.g1 * x.g5 * x.g6) + (-T(32) * x.g2 * x.g5 * x.g6 - T(20) * x.g3 * x.g5 * x.g6 - T(42) * x.g4 * x.g5 * x.g6 - T(17) * x.g5 * x.g5 * x.g6 - T(20) * x.g1 * x.g6 * x.g6 - T(11) * x.g2 * x.g6 * x.g6) + (-T(20) * x.g4 * x.g6 * x.g6 - T(11) * x.g5 * x.g6 * x.g6 + T(16) * x.g2 * x.g7 - T(28) * x.g1 * x.g2 * x.g7 - T(20) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7) + (-T(48) * x.g1 * x.g3 * x.g7 - T(44) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(24) * x.g2 * x.g4 * x.g7 - T(44) * x.g3 * x.g4 * x.g7) + (T(12) * x.g5 * x.g7 - T(28) * x.g1 * x.g5 * x.g7 - T(40) * x.g2 * x.g5 * x.g7 - T(48) * x.g3 * x.g5 * x.g7 - T(20) * x.g4 * x.g5 * x.g7 - T(16) * x.g5 * x.g5 * x.g7) + (T(16) * x.g6 * x.g7 - T(48) * x.g1 * x.g6 * x.g7 - T(48) * x.g2 * x.g6 * x.g7 - T(44) * x.g3 * x.g6 * x.g7 - T(36) * x.g4 * x.g6 * x.g7 - T(40) * x.g5 * x.g6 * x.g7) + (-T(20) * x.g6 * x.g6 * x.g7 - T(8) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - T(4) * x.g5 * x.g7 * x.g7 - T(8) * x.g6 * x.g7 * x.g7 + T(16) * x.g1 * x.g8 - T(8) * x.g1 * x.g1 * x.g8) + (T(24) * x.g2 * x.g8 - T(36) * x.g1 * x.g2 * x.g8 - T(20) * x.g2 * x.g2 * x.g8 + T(16) * x.g3 * x.g8 - T(48) * x.g1 * x.g3 * x.g8 - T(36) * x.g2 * x.g3 * x.g8 - T(8) * x.g3 * x.g3 * x.g8) + (T(13) * x.g4 * x.g8 - T(24) * x.g1 * x.g4 * x.g8 - T(38) * x.g2 * x.g4 * x.g8 - T(48) * x.g3 * x.g4 * x.g8 - T(11) * x.g4 * x.g4 * x.g8 + T(17) * x.g5 * x.g8 - T(40) * x.g1 * x.g5 * x.g8) + (-T(42) * x.g2 * x.g5 * x.g8 - T(40) * x.g3 * x.g5 * x.g8 - T(32) * x.g4 * x.g5 * x.g8 - T(17) * x.g5 * x.g5 * x.g8 + T(13) * x.g6 * x.g8 - T(48) * x.g1 * x.g6 * x.g8) + (-T(38) * x.g2 * x.g6 * x.g8 - T(24) * x.g3 * x.g6 * x.g8 - T(38) * x.g4 * x.g6 * x.g8 - T(32) * x.g5 * x.g6 * x.g8 - T(11) * x.g6 * x.g6 * x.g8 - T(28) * x.g1 * x.g7 * x.g8) + (-T(36) * x.g2 * x.g7 * x.g8 - T(44) * x.g3 * x.g7 * x.g8 - T(16) * x.g4 * x.g7 * x.g8 - T(20) * x.g5 * x.g7 * x.g8 - T(24) * x.g6 * x.g7 * x.g8 - T(20) * x.g1 * x.g8 * x.g8) + (-T(20) * x.g2 * x.g8 * x.g8 - T(20) * x.g3 * x.g8 * x.g8 - T(11) * x.g4 * x.g8 * x.g8 - T(11) * x.g5 * x.g8 * x.g8 - T(11) * x.g6 * x.g8 * x.g8 + T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9) + (T(16) * x.g2 * x.g9 - T(44) * x.g1 * x.g2 * x.g9 - T(20) * x.g2 * x.g2 * x.g9 - T(48) * x.g1 * x.g3 * x.g9 - T(28) * x.g2 * x.g3 * x.g9 + T(16) * x.g4 * x.g9) + (-T(44) * x.g1 * x.g4 * x.g9 - T(48) * x.g2 * x.g4 * x.g9 - T(48) * x.g3 * x.g4 * x.g9 - T(20) * x.g4 * x.g4 * x.g9 + T(12) * x.g5 * x.g9 - T(48) * x.g1 * x.g5 * x.g9) + (-T(40) * x.g2 * x.g5 * x.g9 - T(28) * x.g3 * x.g5 * x.g9 - T(40) * x.g4 * x.g5 * x.g9 - T(16) * x.g5 * x.g5 * x.g9 - T(44) * x.g1 * x.g6 * x.g9 - T(24) * x.g2 * x.g6 * x.g9) + (-T(36) * x.g4 * x.g6 * x.g9 - T(20) * x.g5 * x.g6 * x.g9 - T(48) * x.g1 * x.g7 * x.g9 - T(48) * x.g2 * x.g7 * x.g9 - T(48) * x.g3 * x.g7 * x.g9 - T(28) * x.g4 * x.g7 * x.g9) + (-T(28) * x.g5 * x.g7 * x.g9 - T(28) * x.g6 * x.g7 * x.g9 - T(44) * x.g1 * x.g8 * x.g9 - T(36) * x.g2 * x.g8 * x.g9 - T(28) * x.g3 * x.g8 * x.g9 - T(24) * x.g4 * x.g8 * x.g9) + (-T(20) * x.g5 * x.g8 * x.g9 - T(16) * x.g6 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(8) * x.g2 * x.g9 * x.g9 - T(8) * x.g4 * x.g9 * x.g9 - T(4) * x.g5 * x.g9 * x.g9) ) * T(0.0625)) * x.w4;
}
template <typename T>
LDK_DEV void geno_stats_P1(const GenoFeat<T>* f, T* acc) {
    const T v0 = f[0].DD1;  // dd1(0,)
    const T v1 = f[0].DZ1;  // dz_iii(0,)
    const T v2 = f[0].PI1;  // pi2_same(0,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // Dz_0_0_0
    acc[2] += v2;  // pi2_0_0_0_0
}

// genotype path, P = 2: 15 statistics from 21 distinct raw calls
template <typename T>
LDK_DEV void geno_features_P2(GenoFeat<T>& x) {
    geno_prepare(x);
    x.xAB = x.g1 + T(0.5) * x.g2 + T(0.5) * x.g4 + T(0.25) * x.g5;
    x.xAb = T(0.5) * x.g2 + x.g3 + T(0.25) * x.g5 + T(0.5) * x.g6;
    x.xaB = T(0.5) * x.g4 + T(0.25) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.xab = T(0.25) * x.g5 + T(0.5) * x.g6 + T(0.5) * x.g8 + x.g9;
    x.D = x.xAB * x.xab - x.xAb * x.xaB;
    x.pA = x.g1 + x.g2 + x.g3 + T(0.5) * (x.g4 + x.g5 + x.g6);
    x.qA = T(0.5) * (x.g4 + x.g5 + x.g6) + x.g7 + x.g8 + x.g9;
    x.pB = x.g1 + T(0.5) * x.g2 + x.g4 + T(0.5) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.qB = T(0.5) * x.g2 + x.g3 + T(0.5) * x.g5 + x.g6 + T(0.5) * x.g8 + x.g9;
    x.BL = (T(4) * x.pA * x.qA - (x.g4 + x.g5 + x.g6)) * x.inn1;
    x.BR = (T(4) * x.pB * x.qB - (x.g2 + x.g5 + x.g8)) * x.inn1;
    x.Bsgn = x.xAB - x.xAb - x.xaB + x.xab;
    x.p = x.pA * x.invn;
    x.q = x.pB * x.invn;
    x.L0 = x.g5 + T(2) * x.g6 + T(2) * x.g8 + T(4) * x.g9;
    x.AQ3 = -(x.qB * (T(3) * x.g4 + T(3) * x.g5 + T(3) * x.g6 + T(4) * x.g7 + T(4) * x.g8 + T(4) * x.g9)) / T(8) + x.pA * x.qB * x.qA / T(2) + (x.qA * x.L0) / T(8) + (x.g5 + T(2) * x.g6) / T(8) - (x.pA * x.L0) / T(8);
    x.AS3 = -(x.pB * (T(5) * x.g4 + T(5) * x.g5 + T(5) * x.g6 + T(8) * x.g7 + T(8) * x.g8 + T(8) * x.g9)) / T(8) + x.pA * x.pB * x.qA / T(2) + (x.qA * (-T(2) * x.g2 - T(4) * x.g3 + T(4) * x.g4 + x.g5 - T(2) * x.g6 + T(8) * x.g7 + T(4) * x.g8 + T(4))) / T(8) + (-x.g5 - T(2) * x.g6 - T(4) * x.g7 - T(4) * x.g8 - T(4) * x.g9) / T(8) + (x.pA * x.L0) / T(8);
    x.BP3 = -(x.qA * (T(3) * x.g2 + T(4) * x.g3 + T(3) * x.g5 + T(4) * x.g6 + T(3) * x.g8 + T(4) * x.g9)) / T(8) + x.pB * x.qB * x.qA / T(2) + (x.qB * x.L0) / T(8) + (x.g5 + T(2) * x.g8) / T(8) - (x.pB * x.L0) / T(8);
    x.BR3 = -(x.pA * (T(5) * x.g2 + T(8) * x.g3 + T(5) * x.g5 + T(8) * x.g6 + T(5) * x.g8 + T(8) * x.g9)) / T(8) + x.pA * x.pB * x.qB / T(2) + (x.qB * (T(4) * x.g2 + T(8) * x.g3 - T(2) * x.g4 + x.g5 + T(4) * x.g6 - T(4) * x.g7 - T(2) * x.g8 + T(4))) / T(8) + (-T(4) * x.g3 - x.g5 - T(4) * x.g6 - T(2) * x.g8 - T(4) * x.g9) / T(8) + (x.pB * x.L0) / T(8);
    x.A = -x.g1 + x.g3 - x.g4 + x.g6 - x.g7 + x.g9;
    x.Bv = -x.g1 - x.g2 - x.g3 + x.g7 + x.g8 + x.g9;
    x.Wjj = (-x.g1 + x.g3 + x.g7 - x.g9) + x.A * x.Bv;
    x.U = x.D * (T(1) + x.Bv) + T(0.25) * (T(2) * x.g2 * x.g7 + T(4) * x.g3 * x.g7 + T(2) * x.g5 * x.g7 + T(4) * x.g6 * x.g7 - T(2) * x.g1 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g4 * x.g8 + T(2) * x.g6 * x.g8 - T(4) * x.g1 * x.g9 - T(2) * x.g2 * x.g9 - T(4) * x.g4 * x.g9 - T(2) * x.g5 * x.g9);
    x.V = x.D * (T(1) + x.A) + T(0.25) * (T(2) * x.g3 * x.g4 + T(2) * x.g3 * x.g5 - T(2) * x.g1 * x.g6 - T(2) * x.g2 * x.g6 + T(4) * x.g3 * x.g7 + T(2) * x.g6 * x.g7 + T(4) * x.g3 * x.g8 + T(2) * x.g6 * x.g8 - T(4) * x.g1 * x.g9 - T(4) * x.g2 * x.g9 - T(2) * x.g4 * x.g9 - T(2) * x.g5 * x.g9);
    x.DD1 = T(4) * (((x.g2 * x.g4 - x.g2 * x.g2 * x.g4 + T(4) * x.g3 * x.g4 - T(4) * x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4) + (-x.g2 * x.g4 * x.g4 - T(4) * x.g3 * x.g4 * x.g4) + (x.g1 * x.g5 - x.g1 * x.g1 * x.g5 + x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g3 * x.g3 * x.g5 - T(4) * x.g3 * x.g4 * x.g5 - x.g1 * x.g5 * x.g5 - x.g3 * x.g5 * x.g5) + (T(4) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 + x.g2 * x.g6 - T(4) * x.g1 * x.g2 * x.g6 - x.g2 * x.g2 * x.g6 + T(2) * x.g2 * x.g4 * x.g6 - T(4) * x.g1 * x.g5 * x.g6 - T(4) * x.g1 * x.g6 * x.g6 - x.g2 * x.g6 * x.g6) + (T(4) * x.g2 * x.g7 - T(4) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7 - T(16) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(4) * x.g2 * x.g4 * x.g7 - T(16) * x.g3 * x.g4 * x.g7 + x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 - T(4) * x.g2 * x.g5 * x.g7 - T(18) * x.g3 * x.g5 * x.g7 - x.g5 * x.g5 * x.g7 + T(4) * x.g6 * x.g7 + T(8) * x.g1 * x.g6 * x.g7 - T(16) * x.g3 * x.g6 * x.g7 - T(4) * x.g5 * x.g6 * x.g7 - T(4) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7) + (T(4) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 + T(4) * x.g3 * x.g8 + T(8) * x.g1 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 + x.g4 * x.g8 - T(4) * x.g1 * x.g4 * x.g8 + T(2) * x.g2 * x.g4 * x.g8 - x.g4 * x.g4 * x.g8 - T(4) * x.g1 * x.g5 * x.g8 - T(4) * x.g3 * x.g5 * x.g8 + x.g6 * x.g8 + T(2) * x.g2 * x.g6 * x.g8 - T(4) * x.g3 * x.g6 * x.g8 + T(2) * x.g4 * x.g6 * x.g8 - x.g6 * x.g6 * x.g8 - T(16) * x.g3 * x.g7 * x.g8 - T(4) * x.g6 * x.g7 * x.g8 - T(4) * x.g1 * x.g8 * x.g8 - T(4) * x.g3 * x.g8 * x.g8 - x.g4 * x.g8 * x.g8 - x.g6 * x.g8 * x.g8) + (T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9 + T(4) * x.g2 * x.g9 - T(16) * x.g1 * x.g2 * x.g9 - T(4) * x.g2 * x.g2 * x.g9 + T(4) * x.g4 * x.g9 - T(16) * x.g1 * x.g4 * x.g9 + T(8) * x.g3 * x.g4 * x.g9 - T(4) * x.g4 * x.g4 * x.g9 + x.g5 * x.g9 - T(18) * x.g1 * x.g5 * x.g9 - T(4) * x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 - T(4) * x.g4 * x.g5 * x.g9 - x.g5 * x.g5 * x.g9 - T(16) * x.g1 * x.g6 * x.g9 - T(4) * x.g2 * x.g6 * x.g9 + T(8) * x.g2 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 - T(16) * x.g1 * x.g8 * x.g9 - T(4) * x.g4 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - x.g5 * x.g9 * x.g9) ) * T(0.0625) + x.D * x.D) * x.w4;
    x.DZ1 = T(2) * (T(0.25) * (-(x.g2 * x.g4) + T(3) * x.g1 * x.g2 * x.g4 + x.g2 * x.g2 * x.g4 + T(2) * x.g3 * x.g4 + T(4) * x.g1 * x.g3 * x.g4 - x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4 + x.g2 * x.g4 * x.g4 + T(2) * x.g3 * x.g4 * x.g4 + T(2) * x.g1 * x.g5 - T(3) * x.g1 * x.g1 * x.g5 - x.g1 * x.g2 * x.g5 + T(2) * x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g2 * x.g3 * x.g5 - T(3) * x.g3 * x.g3 * x.g5 - x.g1 * x.g4 * x.g5 + x.g3 * x.g4 * x.g5 + T(2) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 - x.g2 * x.g6 - x.g1 * x.g2 * x.g6 + x.g2 * x.g2 * x.g6 + T(4) * x.g1 * x.g3 * x.g6 + T(3) * x.g2 * x.g3 * x.g6 - T(2) * x.g1 * x.g4 * x.g6 - T(2) * x.g2 * x.g4 * x.g6 - T(2) * x.g3 * x.g4 * x.g6 + x.g1 * x.g5 * x.g6 - x.g3 * x.g5 * x.g6 + T(2) * x.g1 * x.g6 * x.g6 + x.g2 * x.g6 * x.g6 + T(2) * x.g2 * x.g7 + T(4) * x.g1 * x.g2 * x.g7 + T(2) * x.g2 * x.g2 * x.g7 + T(8) * x.g3 * x.g7 + T(4) * x.g1 * x.g3 * x.g7 - T(4) * x.g3 * x.g3 * x.g7 - x.g2 * x.g4 * x.g7 + T(2) * x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 + x.g2 * x.g5 * x.g7 + T(2) * x.g3 * x.g5 * x.g7 - x.g4 * x.g5 * x.g7 + T(2) * x.g6 * x.g7 - x.g2 * x.g6 * x.g7 - T(2) * x.g4 * x.g6 * x.g7 + x.g5 * x.g6 * x.g7 + T(2) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(4) * x.g3 * x.g7 * x.g7 - T(3) * x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7 + T(2) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 - T(2) * x.g1 * x.g2 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g2 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 - x.g4 * x.g8 - x.g1 * x.g4 * x.g8 - T(2) * x.g2 * x.g4 * x.g8 - x.g3 * x.g4 * x.g8 + x.g4 * x.g4 * x.g8 + x.g1 * x.g5 * x.g8 + x.g3 * x.g5 * x.g8 - x.g6 * x.g8 - x.g1 * x.g6 * x.g8 - T(2) * x.g2 * x.g6 * x.g8 - x.g3 * x.g6 * x.g8 - T(2) * x.g4 * x.g6 * x.g8 + x.g6 * x.g6 * x.g8 + T(4) * x.g1 * x.g7 * x.g8 - T(2) * x.g2 * x.g7 * x.g8 + T(3) * x.g4 * x.g7 * x.g8 - x.g5 * x.g7 * x.g8 - x.g6 * x.g7 * x.g8 + T(2) * x.g1 * x.g8 * x.g8 + T(2) * x.g3 * x.g8 * x.g8 + x.g4 * x.g8 * x.g8 + x.g6 * x.g8 * x.g8 + T(8) * x.g1 * x.g9 - T(4) * x.g1 * x.g1 * x.g9 + T(2) * x.g2 * x.g9 + T(2) * x.g2 * x.g2 * x.g9 + T(4) * x.g1 * x.g3 * x.g9 + T(4) * x.g2 * x.g3 * x.g9 + T(2) * x.g4 * x.g9 - x.g2 * x.g4 * x.g9 + T(2) * x.g4 * x.g4 * x.g9 + T(2) * x.g5 * x.g9 + T(2) * x.g1 * x.g5 * x.g9 + x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 + x.g4 * x.g5 * x.g9 - x.g2 * x.g6 * x.g9 - T(2) * x.g4 * x.g6 * x.g9 - x.g5 * x.g6 * x.g9 + T(4) * x.g1 * x.g7 * x.g9 + T(4) * x.g3 * x.g7 * x.g9 + T(4) * x.g4 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 + T(4) * x.g6 * x.g7 * x.g9 - T(2) * x.g2 * x.g8 * x.g9 + T(4) * x.g3 * x.g8 * x.g9 - x.g4 * x.g8 * x.g9 - x.g5 * x.g8 * x.g9 + T(3) * x.g6 * x.g8 * x.g9 - T(4) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - T(3) * x.g5 * x.g9 * x.g9 ) + x.A * x.Bv * x.D) * x.w4;
    x.PI1 = (x.pA * x.pB * x.qB * x.qA + ((T(13) * x.g2 * x.g4 - T(16) * x.g1 * x.g2 * x.g4 - T(11) * x.g2 * x.g2 * x.g4 + T(16) * x.g3 * x.g4 - T(28) * x.g1 * x.g3 * x.g4 - T(24) * x.g2 * x.g3 * x.g4) + (-T(8) * x.g3 * x.g3 * x.g4 - T(11) * x.g2 * x.g4 * x.g4 - T(20) * x.g3 * x.g4 * x.g4 - T(6) * x.g5 + T(12) * x.g1 * x.g5 - T(4) * x.g1 * x.g1 * x.g5 + T(17) * x.g2 * x.g5) + (-T(20) * x.g1 * x.g2 * x.g5 - T(11) * x.g2 * x.g2 * x.g5 + T(12) * x.g3 * x.g5 - T(28) * x.g1 * x.g3 * x.g5 - T(20) * x.g2 * x.g3 * x.g5 - T(4) * x.g3 * x.g3 * x.g5) + (T(17) * x.g4 * x.g5 - T(20) * x.g1 * x.g4 * x.g5 - T(32) * x.g2 * x.g4 * x.g5 - T(40) * x.g3 * x.g4 * x.g5 - T(11) * x.g4 * x.g4 * x.g5 + T(11) * x.g5 * x.g5) + (-T(16) * x.g1 * x.g5 * x.g5 - T(17) * x.g2 * x.g5 * x.g5 - T(16) * x.g3 * x.g5 * x.g5 - T(17) * x.g4 * x.g5 * x.g5 - T(6) * x.g5 * x.g5 * x.g5 + T(16) * x.g1 * x.g6 - T(8) * x.g1 * x.g1 * x.g6) + (T(13) * x.g2 * x.g6 - T(24) * x.g1 * x.g2 * x.g6 - T(11) * x.g2 * x.g2 * x.g6 - T(28) * x.g1 * x.g3 * x.g6 - T(16) * x.g2 * x.g3 * x.g6 + T(24) * x.g4 * x.g6) + (-T(36) * x.g1 * x.g4 * x.g6 - T(38) * x.g2 * x.g4 * x.g6 - T(36) * x.g3 * x.g4 * x.g6 - T(20) * x.g4 * x.g4 * x.g6 + T(17) * x.g5 * x.g6 - T(40) * x.g1 * x.g5 * x.g6) + (-T(32) * x.g2 * x.g5 * x.g6 - T(20) * x.g3 * x.g5 * x.g6 - T(42) * x.g4 * x.g5 * x.g6 - T(17) * x.g5 * x.g5 * x.g6 - T(20) * x.g1 * x.g6 * x.g6 - T(11) * x.g2 * x.g6 * x.g6) + (-T(20) * x.g4 * x.g6 * x.g6 - T(11) * x.g5 * x.g6 * x.g6 + T(16) * x.g2 * x.g7 - T(28) * x.g1 * x.g2 * x.g7 - T(20) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7) + (-T(48) * x.g1 * x.g3 * x.g7 - T(44) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(24) * x.g2 * x.g4 * x.g7 - T(44) * x.g3 * x.g4 * x.g7) + (T(12) * x.g5 * x.g7 - T(28) * x.g1 * x.g5 * x.g7 - T(40) * x.g2 * x.g5 * x.g7 - T(48) * x.g3 * x.g5 * x.g7 - T(20) * x.g4 * x.g5 * x.g7 - T(16) * x.g5 * x.g5 * x.g7) + (T(16) * x.g6 * x.g7 - T(48) * x.g1 * x.g6 * x.g7 - T(48) * x.g2 * x.g6 * x.g7 - T(44) * x.g3 * x.g6 * x.g7 - T(36) * x.g4 * x.g6 * x.g7 - T(40) * x.g5 * x.g6 * x.g7) + (-T(20) * x.g6 * x.g6 * x.g7 - T(8) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - T(4) * x.g5 * x.g7 * x.g7 - T(8) * x.g6 * x.g7 * x.g7 + T(16) * x.g1 * x.g8 - T(8) * x.g1 * x.g1 * x.g8) + (T(24) * x.g2 * x.g8 - T(36) * x.g1 * x.g2 * x.g8 - T(20) * x.g2 * x.g2 * x.g8 + T(16) * x.g3 * x.g8 - T(48) * x.g1 * x.g3 * x.g8 - T(36) * x.g2 * x.g3 * x.g8 - T(8) * x.g3 * x.g3 * x.g8) + (T(13) * x.g4 * x.g8 - T(24) * x.g1 * x.g4 * x.g8 - T(38) * x.g2 * x.g4 * x.g8 - T(48) * x.g3 * x.g4 * x.g8 - T(11) * x.g4 * x.g4 * x.g8 + T(17) * x.g5 * x.g8 - T(40) * x.g1 * x.g5 * x.g8) + (-T(42) * x.g2 * x.g5 * x.g8 - T(40) * x.g3 * x.g5 * x.g8 - T(32) * x.g4 * x.g5 * x.g8 - T(17) * x.g5 * x.g5 * x.g8 + T(13) * x.g6 * x.g8 - T(48) * x.g1 * x.g6 * x.g8) + (-T(38) * x.g2 * x.g6 * x.g8 - T(24) * x.g3 * x.g6 * x.g8 - T(38) * x.g4 * x.g6 * x.g8 - T(32) * x.g5 * x.g6 * x.g8 - T(11) * x.g6 * x.g6 * x.g8 - T(28) * x.g1 * x.g7 * x.g8) + (-T(36) * x.g2 * x.g7 * x.g8 - T(44) * x.g3 * x.g7 * x.g8 - T(16) * x.g4 * x.g7 * x.g8 - T(20) * x.g5 * x.g7 * x.g8 - T(24) * x.g6 * x.g7 * x.g8 - T(20) * x.g1 * x.g8 * x.g8) + (-T(20) * x.g2 * x.g8 * x.g8 - T(20) * x.g3 * x.g8 * x.g8 - T(11) * x.g4 * x.g8 * x.g8 - T(11) * x.g5 * x.g8 * x.g8 - T(11) * x.g6 * x.g8 * x.g8 + T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9) + (T(16) * x.g2 * x.g9 - T(44) * x.g1 * x.g2 * x.g9 - T(20) * x.g2 * x.g2 * x.g9 - T(48) * x.g1 * x.g3 * x.g9 - T(28) * x.g2 * x.g3 * x.g9 + T(16) * x.g4 * x.g9) + (-T(44) * x.g1 * x.g4 * x.g9 - T(48) * x.g2 * x.g4 * x.g9 - T(48) * x.g3 * x.g4 * x.g9 - T(20) * x.g4 * x.g4 * x.g9 + T(12) * x.g5 * x.g9 - T(48) * x.g1 * x.g5 * x.g9) + (-T(40) * x.g2 * x.g5 * x.g9 - T(28) * x.g3 * x.g5 * x.g9 - T(40) * x.g4 * x.g5 * x.g9 - T(16) * x.g5 * x.g5 * x.g9 - T(44) * x.g1 * x.g6 * x.g9 - T(24) * x.g2 * x.g6 * x.g9) + (-T(36) * x.g4 * x.g6 * x.g9 - T(20) * x.g5 * x.g6 * x.g9 - T(48) * x.g1 * x.g7 * x.g9 - T(48) * x.g2 * x.g7 * x.g9 - T(48) * x.g3 * x.g7 * x.g9 - T(28) * x.g4 * x.g7 * x.g9) + (-T(28) * x.g5 * x.g7 * x.g9 - T(28) * x.g6 * x.g7 * x.g9 - T(44) * x.g1 * x.g8 * x.g9 - T(36) * x.g2 * x.g8 * x.g9 - T(28) * x.g3 * x.g8 * x.g9 - T(24) * x.g4 * x.g8 * x.g9) + (-T(20) * x.g5 * x.g8 * x.g9 - T(16) * x.g6 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(8) * x.g2 * x.g9 * x.g9 - T(8) * x.g4 * x.g9 * x.g9 - T(4) * x.g5 * x.g9 * x.g9) ) * T(0.0625)) * x.w4;
}
template <typename T>
LDK_DEV void geno_stats_P2(const GenoFeat<T>* f, T* acc) {
    const T v0 = f[0].DD1;  // dd1(0,)
    const T v1 = T(4) * (f[0].D * f[1].D) * (f[0].r2 * f[1].r2);  // dd2(0, 1)
    const T v2 = f[1].DD1;  // dd1(1,)
    const T v3 = f[0].DZ1;  // dz_iii(0,)
    const T v4 = (T(2) * f[0].U * f[1].A) * (f[0].u3 * f[1].u1);  // dz_iij(0, 1)
    const T v5 = (T(2) * f[0].V * f[1].Bv) * (f[0].u3 * f[1].u1);  // dz_iji(0, 1)
    const T v6 = (T(2) * f[0].D * f[1].Wjj) * (f[1].u2 * f[0].u2);  // dz_ijj(0, 1)
    const T v7 = (T(2) * f[1].D * f[0].Wjj) * (f[0].u2 * f[1].u2);  // dz_ijj(1, 0)
    const T v8 = (T(2) * f[1].V * f[0].Bv) * (f[1].u3 * f[0].u1);  // dz_iji(1, 0)
    const T v9 = (T(2) * f[1].U * f[0].A) * (f[1].u3 * f[0].u1);  // dz_iij(1, 0)
    const T v10 = f[1].DZ1;  // dz_iii(1,)
    const T v11 = f[0].PI1;  // pi2_same(0,)
    const T v12 = (f[0].AQ3 * f[1].pB + f[0].AS3 * f[1].qB) * (f[0].r3 * f[1].r1);  // pi2_iiij(0, 1)
    const T v13 = (f[0].BP3 * f[1].pA + f[0].BR3 * f[1].qA) * (f[0].r3 * f[1].r1);  // pi2_ijii(0, 1)
    const T v14 = f[0].BL * f[1].BR;  // pi2_iikk(0, 1)
    const T v15 = f[1].BL * f[0].BR;  // pi2_iikk(1, 0)
    const T v16 = (-T(0.25) * (f[0].qA * f[0].qB) * f[1].pB - T(0.25) * f[0].xab * (f[1].pA * f[1].pB) + T(0.25) * (f[0].qA * f[0].qB) * (f[1].pA * f[1].pB) - T(0.25) * f[0].qA * (f[1].pA * f[1].qB) - T(0.25) * (f[0].pA * f[0].pB) * f[1].xab - T(0.25) * (f[0].qA * f[0].qB) * f[1].xab + T(0.25) * (f[0].pA * f[0].qB) * f[1].xab + T(0.25) * (f[0].pB * f[0].qA) * f[1].xab - T(0.25) * (f[0].pA * f[0].qA) * f[1].qB + T(0.25) * (f[0].qA * (T(1) + f[0].xAb - f[0].xaB)) * f[1].qB + T(0.25) * f[0].xab * (f[1].pA * f[1].qB) + T(0.25) * (f[0].pB * f[0].qA) * (f[1].pA * f[1].qB) + T(0.25) * (f[0].qB * (T(1) + f[0].qA)) * f[1].qA - T(0.25) * f[0].xAb * (f[1].pB * f[1].qA) + T(0.25) * (f[0].pA * f[0].qB) * (f[1].pB * f[1].qA) - T(0.25) * (f[0].pA * f[0].qB) * f[1].qA - T(0.25) * f[0].pA * (f[1].qA * f[1].qB) + T(0.25) * f[0].xAb * (f[1].qA * f[1].qB) + T(0.25) * (f[0].pA * f[0].pB) * (f[1].qA * f[1].qB) + T(0.25) * f[0].xab * f[1].Bsgn + T(0.25) * f[0].Bsgn * f[1].xab - f[0].xab * f[1].xab) * (f[0].r2 * f[1].r2);  // pi2_ijij(0, 1)
    const T v17 = (-T(0.25) * (f[1].qA * f[1].qB) * f[0].pB - T(0.25) * f[1].xab * (f[0].pA * f[0].pB) + T(0.25) * (f[1].qA * f[1].qB) * (f[0].pA * f[0].pB) - T(0.25) * f[1].qA * (f[0].pA * f[0].qB) - T(0.25) * (f[1].pA * f[1].pB) * f[0].xab - T(0.25) * (f[1].qA * f[1].qB) * f[0].xab + T(0.25) * (f[1].pA * f[1].qB) * f[0].xab + T(0.25) * (f[1].pB * f[1].qA) * f[0].xab - T(0.25) * (f[1].pA * f[1].qA) * f[0].qB + T(0.25) * (f[1].qA * (T(1) + f[1].xAb - f[1].xaB)) * f[0].qB + T(0.25) * f[1].xab * (f[0].pA * f[0].qB) + T(0.25) * (f[1].pB * f[1].qA) * (f[0].pA * f[0].qB) + T(0.25) * (f[1].qB * (T(1) + f[1].qA)) * f[0].qA - T(0.25) * f[1].xAb * (f[0].pB * f[0].qA) + T(0.25) * (f[1].pA * f[1].qB) * (f[0].pB * f[0].qA) - T(0.25) * (f[1].pA * f[1].qB) * f[0].qA - T(0.25) * f[1].pA * (f[0].qA * f[0].qB) + T(0.25) * f[1].xAb * (f[0].qA * f[0].qB) + T(0.25) * (f[1].pA * f[1].pB) * (f[0].qA * f[0].qB) + T(0.25) * f[1].xab * f[0].Bsgn + T(0.25) * f[1].Bsgn * f[0].xab - f[1].xab * f[0].xab) * (f[1].r2 * f[0].r2);  // pi2_ijij(1, 0)
    const T v18 = (f[1].BP3 * f[0].pA + f[1].BR3 * f[0].qA) * (f[1].r3 * f[0].r1);  // pi2_ijii(1, 0)
    const T v19 = (f[1].AQ3 * f[0].pB + f[1].AS3 * f[0].qB) * (f[1].r3 * f[0].r1);  // pi2_iiij(1, 0)
    const T v20 = f[1].PI1;  // pi2_same(1,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // DD_0_1
    acc[2] += v2;  // DD_1_1
    acc[3] += v3;  // Dz_0_0_0
    acc[4] += T(0.5) * (v4 + v5);  // Dz_0_0_1
    acc[5] += v6;  // Dz_0_1_1
    acc[6] += v7;  // Dz_1_0_0
    acc[7] += T(0.5) * (v8 + v9);  // Dz_1_0_1
    acc[8] += v10;  // Dz_1_1_1
    acc[9] += v11;  // pi2_0_0_0_0
    acc[10] += T(0.5) * (v12 + v13);  // pi2_0_0_0_1
    acc[11] += T(0.5) * (v14 + v15);  // pi2_0_0_1_1
    acc[12] += T(0.5) * (v16 + v17);  // pi2_0_1_0_1
    acc[13] += T(0.5) * (v18 + v19);  // pi2_0_1_1_1
    acc[14] += v20;  // pi2_1_1_1_1
}

// genotype path, P = 3: 45 statistics from 72 distinct raw calls
template <typename T>
LDK_DEV void geno_features_P3(GenoFeat<T>& x) {
    geno_prepare(x);
    x.xAB = x.g1 + T(0.5) * x.g2 + T(0.5) * x.g4 + T(0.25) * x.g5;
    x.xAb = T(0.5) * x.g2 + x.g3 + T(0.25) * x.g5 + T(0.5) * x.g6;
    x.xaB = T(0.5) * x.g4 + T(0.25) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.xab = T(0.25) * x.g5 + T(0.5) * x.g6 + T(0.5) * x.g8 + x.g9;
    x.D = x.xAB * x.xab - x.xAb * x.xaB;
    x.pA = x.g1 + x.g2 + x.g3 + T(0.5) * (x.g4 + x.g5 + x.g6);
    x.qA = T(0.5) * (x.g4 + x.g5 + x.g6) + x.g7 + x.g8 + x.g9;
    x.pB = x.g1 + T(0.5) * x.g2 + x.g4 + T(0.5) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.qB = T(0.5) * x.g2 + x.g3 + T(0.5) * x.g5 + x.g6 + T(0.5) * x.g8 + x.g9;
    x.BL = (T(4) * x.pA * x.qA - (x.g4 + x.g5 + x.g6)) * x.inn1;
    x.BR = (T(4) * x.pB * x.qB - (x.g2 + x.g5 + x.g8)) * x.inn1;
    x.C00 = (x.pA * x.pB - x.xAB) * x.inn1;
    x.C01 = (x.pA * x.qB - x.xAb) * x.inn1;
    x.C10 = (x.qA * x.pB - x.xaB) * x.inn1;
    x.C11 = (x.qA * x.qB - x.xab) * x.inn1;
    x.Bsgn = x.xAB - x.xAb - x.xaB + x.xab;
    x.p = x.pA * x.invn;
    x.r = x.qA * x.invn;
    x.q = x.pB * x.invn;
    x.s = x.qB * x.invn;
    x.L0 = x.g5 + T(2) * x.g6 + T(2) * x.g8 + T(4) * x.g9;
    x.AQ3 = -(x.qB * (T(3) * x.g4 + T(3) * x.g5 + T(3) * x.g6 + T(4) * x.g7 + T(4) * x.g8 + T(4) * x.g9)) / T(8) + x.pA * x.qB * x.qA / T(2) + (x.qA * x.L0) / T(8) + (x.g5 + T(2) * x.g6) / T(8) - (x.pA * x.L0) / T(8);
    x.AS3 = -(x.pB * (T(5) * x.g4 + T(5) * x.g5 + T(5) * x.g6 + T(8) * x.g7 + T(8) * x.g8 + T(8) * x.g9)) / T(8) + x.pA * x.pB * x.qA / T(2) + (x.qA * (-T(2) * x.g2 - T(4) * x.g3 + T(4) * x.g4 + x.g5 - T(2) * x.g6 + T(8) * x.g7 + T(4) * x.g8 + T(4))) / T(8) + (-x.g5 - T(2) * x.g6 - T(4) * x.g7 - T(4) * x.g8 - T(4) * x.g9) / T(8) + (x.pA * x.L0) / T(8);
    x.BP3 = -(x.qA * (T(3) * x.g2 + T(4) * x.g3 + T(3) * x.g5 + T(4) * x.g6 + T(3) * x.g8 + T(4) * x.g9)) / T(8) + x.pB * x.qB * x.qA / T(2) + (x.qB * x.L0) / T(8) + (x.g5 + T(2) * x.g8) / T(8) - (x.pB * x.L0) / T(8);
    x.BR3 = -(x.pA * (T(5) * x.g2 + T(8) * x.g3 + T(5) * x.g5 + T(8) * x.g6 + T(5) * x.g8 + T(8) * x.g9)) / T(8) + x.pA * x.pB * x.qB / T(2) + (x.qB * (T(4) * x.g2 + T(8) * x.g3 - T(2) * x.g4 + x.g5 + T(4) * x.g6 - T(4) * x.g7 - T(2) * x.g8 + T(4))) / T(8) + (-T(4) * x.g3 - x.g5 - T(4) * x.g6 - T(2) * x.g8 - T(4) * x.g9) / T(8) + (x.pB * x.L0) / T(8);
    x.A = -x.g1 + x.g3 - x.g4 + x.g6 - x.g7 + x.g9;
    x.Bv = -x.g1 - x.g2 - x.g3 + x.g7 + x.g8 + x.g9;
    x.Wjj = (-x.g1 + x.g3 + x.g7 - x.g9) + x.A * x.Bv;
    x.U = x.D * (T(1) + x.Bv) + T(0.25) * (T(2) * x.g2 * x.g7 + T(4) * x.g3 * x.g7 + T(2) * x.g5 * x.g7 + T(4) * x.g6 * x.g7 - T(2) * x.g1 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g4 * x.g8 + T(2) * x.g6 * x.g8 - T(4) * x.g1 * x.g9 - T(2) * x.g2 * x.g9 - T(4) * x.g4 * x.g9 - T(2) * x.g5 * x.g9);
    x.V = x.D * (T(1) + x.A) + T(0.25) * (T(2) * x.g3 * x.g4 + T(2) * x.g3 * x.g5 - T(2) * x.g1 * x.g6 - T(2) * x.g2 * x.g6 + T(4) * x.g3 * x.g7 + T(2) * x.g6 * x.g7 + T(4) * x.g3 * x.g8 + T(2) * x.g6 * x.g8 - T(4) * x.g1 * x.g9 - T(4) * x.g2 * x.g9 - T(2) * x.g4 * x.g9 - T(2) * x.g5 * x.g9);
    x.DD1 = T(4) * (((x.g2 * x.g4 - x.g2 * x.g2 * x.g4 + T(4) * x.g3 * x.g4 - T(4) * x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4) + (-x.g2 * x.g4 * x.g4 - T(4) * x.g3 * x.g4 * x.g4) + (x.g1 * x.g5 - x.g1 * x.g1 * x.g5 + x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g3 * x.g3 * x.g5 - T(4) * x.g3 * x.g4 * x.g5 - x.g1 * x.g5 * x.g5 - x.g3 * x.g5 * x.g5) + (T(4) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 + x.g2 * x.g6 - T(4) * x.g1 * x.g2 * x.g6 - x.g2 * x.g2 * x.g6 + T(2) * x.g2 * x.g4 * x.g6 - T(4) * x.g1 * x.g5 * x.g6 - T(4) * x.g1 * x.g6 * x.g6 - x.g2 * x.g6 * x.g6) + (T(4) * x.g2 * x.g7 - T(4) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7 - T(16) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(4) * x.g2 * x.g4 * x.g7 - T(16) * x.g3 * x.g4 * x.g7 + x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 - T(4) * x.g2 * x.g5 * x.g7 - T(18) * x.g3 * x.g5 * x.g7 - x.g5 * x.g5 * x.g7 + T(4) * x.g6 * x.g7 + T(8) * x.g1 * x.g6 * x.g7 - T(16) * x.g3 * x.g6 * x.g7 - T(4) * x.g5 * x.g6 * x.g7 - T(4) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7) + (T(4) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 + T(4) * x.g3 * x.g8 + T(8) * x.g1 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 + x.g4 * x.g8 - T(4) * x.g1 * x.g4 * x.g8 + T(2) * x.g2 * x.g4 * x.g8 - x.g4 * x.g4 * x.g8 - T(4) * x.g1 * x.g5 * x.g8 - T(4) * x.g3 * x.g5 * x.g8 + x.g6 * x.g8 + T(2) * x.g2 * x.g6 * x.g8 - T(4) * x.g3 * x.g6 * x.g8 + T(2) * x.g4 * x.g6 * x.g8 - x.g6 * x.g6 * x.g8 - T(16) * x.g3 * x.g7 * x.g8 - T(4) * x.g6 * x.g7 * x.g8 - T(4) * x.g1 * x.g8 * x.g8 - T(4) * x.g3 * x.g8 * x.g8 - x.g4 * x.g8 * x.g8 - x.g6 * x.g8 * x.g8) + (T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9 + T(4) * x.g2 * x.g9 - T(16) * x.g1 * x.g2 * x.g9 - T(4) * x.g2 * x.g2 * x.g9 + T(4) * x.g4 * x.g9 - T(16) * x.g1 * x.g4 * x.g9 + T(8) * x.g3 * x.g4 * x.g9 - T(4) * x.g4 * x.g4 * x.g9 + x.g5 * x.g9 - T(18) * x.g1 * x.g5 * x.g9 - T(4) * x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 - T(4) * x.g4 * x.g5 * x.g9 - x.g5 * x.g5 * x.g9 - T(16) * x.g1 * x.g6 * x.g9 - T(4) * x.g2 * x.g6 * x.g9 + T(8) * x.g2 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 - T(16) * x.g1 * x.g8 * x.g9 - T(4) * x.g4 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - x.g5 * x.g9 * x.g9) ) * T(0.0625) + x.D * x.D) * x.w4;
    x.DZ1 = T(2) * (T(0.25) * (-(x.g2 * x.g4) + T(3) * x.g1 * x.g2 * x.g4 + x.g2 * x.g2 * x.g4 + T(2) * x.g3 * x.g4 + T(4) * x.g1 * x.g3 * x.g4 - x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4 + x.g2 * x.g4 * x.g4 + T(2) * x.g3 * x.g4 * x.g4 + T(2) * x.g1 * x.g5 - T(3) * x.g1 * x.g1 * x.g5 - x.g1 * x.g2 * x.g5 + T(2) * x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g2 * x.g3 * x.g5 - T(3) * x.g3 * x.g3 * x.g5 - x.g1 * x.g4 * x.g5 + x.g3 * x.g4 * x.g5 + T(2) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 - x.g2 * x.g6 - x.g1 * x.g2 * x.g6 + x.g2 * x.g2 * x.g6 + T(4) * x.g1 * x.g3 * x.g6 + T(3) * x.g2 * x.g3 * x.g6 - T(2) * x.g1 * x.g4 * x.g6 - T(2) * x.g2 * x.g4 * x.g6 - T(2) * x.g3 * x.g4 * x.g6 + x.g1 * x.g5 * x.g6 - x.g3 * x.g5 * x.g6 + T(2) * x.g1 * x.g6 * x.g6 + x.g2 * x.g6 * x.g6 + T(2) * x.g2 * x.g7 + T(4) * x.g1 * x.g2 * x.g7 + T(2) * x.g2 * x.g2 * x.g7 + T(8) * x.g3 * x.g7 + T(4) * x.g1 * x.g3 * x.g7 - T(4) * x.g3 * x.g3 * x.g7 - x.g2 * x.g4 * x.g7 + T(2) * x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 + x.g2 * x.g5 * x.g7 + T(2) * x.g3 * x.g5 * x.g7 - x.g4 * x.g5 * x.g7 + T(2) * x.g6 * x.g7 - x.g2 * x.g6 * x.g7 - T(2) * x.g4 * x.g6 * x.g7 + x.g5 * x.g6 * x.g7 + T(2) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(4) * x.g3 * x.g7 * x.g7 - T(3) * x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7 + T(2) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 - T(2) * x.g1 * x.g2 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g2 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 - x.g4 * x.g8 - x.g1 * x.g4 * x.g8 - T(2) * x.g2 * x.g4 * x.g8 - x.g3 * x.g4 * x.g8 + x.g4 * x.g4 * x.g8 + x.g1 * x.g5 * x.g8 + x.g3 * x.g5 * x.g8 - x.g6 * x.g8 - x.g1 * x.g6 * x.g8 - T(2) * x.g2 * x.g6 * x.g8 - x.g3 * x.g6 * x.g8 - T(2) * x.g4 * x.g6 * x.g8 + x.g6 * x.g6 * x.g8 + T(4) * x.g1 * x.g7 * x.g8 - T(2) * x.g2 * x.g7 * x.g8 + T(3) * x.g4 * x.g7 * x.g8 - x.g5 * x.g7 * x.g8 - x.g6 * x.g7 * x.g8 + T(2) * x.g1 * x.g8 * x.g8 + T(2) * x.g3 * x.g8 * x.g8 + x.g4 * x.g8 * x.g8 + x.g6 * x.g8 * x.g8 + T(8) * x.g1 * x.g9 - T(4) * x.g1 * x.g1 * x.g9 + T(2) * x.g2 * x.g9 + T(2) * x.g2 * x.g2 * x.g9 + T(4) * x.g1 * x.g3 * x.g9 + T(4) * x.g2 * x.g3 * x.g9 + T(2) * x.g4 * x.g9 - x.g2 * x.g4 * x.g9 + T(2) * x.g4 * x.g4 * x.g9 + T(2) * x.g5 * x.g9 + T(2) * x.g1 * x.g5 * x.g9 + x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 + x.g4 * x.g5 * x.g9 - x.g2 * x.g6 * x.g9 - T(2) * x.g4 * x.g6 * x.g9 - x.g5 * x.g6 * x.g9 + T(4) * x.g1 * x.g7 * x.g9 + T(4) * x.g3 * x.g7 * x.g9 + T(4) * x.g4 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 + T(4) * x.g6 * x.g7 * x.g9 - T(2) * x.g2 * x.g8 * x.g9 + T(4) * x.g3 * x.g8 * x.g9 - x.g4 * x.g8 * x.g9 - x.g5 * x.g8 * x.g9 + T(3) * x.g6 * x.g8 * x.g9 - T(4) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - T(3) * x.g5 * x.g9 * x.g9 ) + x.A * x.Bv * x.D) * x.w4;
    x.PI1 = (x.pA * x.pB * x.qB * x.qA + ((T(13) * x.g2 * x.g4 - T(16) * x.g1 * x.g2 * x.g4 - T(11) * x.g2 * x.g2 * x.g4 + T(16) * x.g3 * x.g4 - T(28) * x.g1 * x.g3 * x.g4 - T(24) * x.g2 * x.g3 * x.g4) + (-T(8) * x.g3 * x.g3 * x.g4 - T(11) * x.g2 * x.g4 * x.g4 - T(20) * x.g3 * x.g4 * x.g4 - T(6) * x.g5 + T(12) * x.g1 * x.g5 - T(4) * x.g1 * x.g1 * x.g5 + T(17) * x.g2 * x.g5) + (-T(20) * x.g1 * x.g2 * x.g5 - T(11) * x.g2 * x.g2 * x.g5 + T(12) * x.g3 * x.g5 - T(28) * x.g1 * x.g3 * x.g5 - T(20) * x.g2 * x.g3 * x.g5 - T(4) * x.g3 * x.g3 * x.g5) + (T(17) * x.g4 * x.g5 - T(20) * x.g1 * x.g4 * x.g5 - T(32) * x.g2 * x.g4 * x.g5 - T(40) * x.g3 * x.g4 * x.g5 - T(11) * x.g4 * x.g4 * x.g5 + T(11) * x.g5 * x.g5) + (-T(16) * x.g1 * x.g5 * x.g5 - T(17) * x.g2 * x.g5 * x.g5 - T(16) * x.g3 * x.g5 * x.g5 - T(17) * x.g4 * x.g5 * x.g5 - T(6) * x.g5 * x.g5 * x.g5 + T(16) * x.g1 * x.g6 - T(8) * x.g1 * x.g1 * x.g6) + (T(13) * x.g2 * x.g6 - T(24) * x.g1 * x.g2 * x.g6 - T(11) * x.g2 * x.g2 * x.g6 - T(28) * x.g1 * x.g3 * x.g6 - T(16) * x.g2 * x.g3 * x.g6 + T(24) * x.g4 * x.g6) + (-T(36) * x.g1 * x.g4 * x.g6 - T(38) * x.g2 * x.g4 * x.g6 - T(36) * x.g3 * x.g4 * x.g6 - T(20) * x.g4 * x.g4 * x.g6 + T(17) * x.g5 * x.g6 - T(40) * x.g1 * x.g5 * x.g6) + (-T(32) * x.g2 * x.g5 * x.g6 - T(20) * x.g3 * x.g5 * x.g6 - T(42) * x.g4 * x.g5 * x.g6 - T(17) * x.g5 * x.g5 * x.g6 - T(20) * x.g1 * x.g6 * x.g6 - T(11) * x.g2 * x.g6 * x.g6) + (-T(20) * x.g4 * x.g6 * x.g6 - T(11) * x.g5 * x.g6 * x.g6 + T(16) * x.g2 * x.g7 - T(28) * x.g1 * x.g2 * x.g7 - T(20) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7) + (-T(48) * x.g1 * x.g3 * x.g7 - T(44) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(24) * x.g2 * x.g4 * x.g7 - T(44) * x.g3 * x.g4 * x.g7) + (T(12) * x.g5 * x.g7 - T(28) * x.g1 * x.g5 * x.g7 - T(40) * x.g2 * x.g5 * x.g7 - T(48) * x.g3 * x.g5 * x.g7 - T(20) * x.g4 * x.g5 * x.g7 - T(16) * x.g5 * x.g5 * x.g7) + (T(16) * x.g6 * x.g7 - T(48) * x.g1 * x.g6 * x.g7 - T(48) * x.g2 * x.g6 * x.g7 - T(44) * x.g3 * x.g6 * x.g7 - T(36) * x.g4 * x.g6 * x.g7 - T(40) * x.g5 * x.g6 * x.g7) + (-T(20) * x.g6 * x.g6 * x.g7 - T(8) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - T(4) * x.g5 * x.g7 * x.g7 - T(8) * x.g6 * x.g7 * x.g7 + T(16) * x.g1 * x.g8 - T(8) * x.g1 * x.g1 * x.g8) + (T(24) * x.g2 * x.g8 - T(36) * x.g1 * x.g2 * x.g8 - T(20) * x.g2 * x.g2 * x.g8 + T(16) * x.g3 * x.g8 - T(48) * x.g1 * x.g3 * x.g8 - T(36) * x.g2 * x.g3 * x.g8 - T(8) * x.g3 * x.g3 * x.g8) + (T(13) * x.g4 * x.g8 - T(24) * x.g1 * x.g4 * x.g8 - T(38) * x.g2 * x.g4 * x.g8 - T(48) * x.g3 * x.g4 * x.g8 - T(11) * x.g4 * x.g4 * x.g8 + T(17) * x.g5 * x.g8 - T(40) * x.g1 * x.g5 * x.g8) + (-T(42) * x.g2 * x.g5 * x.g8 - T(40) * x.g3 * x.g5 * x.g8 - T(32) * x.g4 * x.g5 * x.g8 - T(17) * x.g5 * x.g5 * x.g8 + T(13) * x.g6 * x.g8 - T(48) * x.g1 * x.g6 * x.g8) + (-T(38) * x.g2 * x.g6 * x.g8 - T(24) * x.g3 * x.g6 * x.g8 - T(38) * x.g4 * x.g6 * x.g8 - T(32) * x.g5 * x.g6 * x.g8 - T(11) * x.g6 * x.g6 * x.g8 - T(28) * x.g1 * x.g7 * x.g8) + (-T(36) * x.g2 * x.g7 * x.g8 - T(44) * x.g3 * x.g7 * x.g8 - T(16) * x.g4 * x.g7 * x.g8 - T(20) * x.g5 * x.g7 * x.g8 - T(24) * x.g6 * x.g7 * x.g8 - T(20) * x.g1 * x.g8 * x.g8) + (-T(20) * x.g2 * x.g8 * x.g8 - T(20) * x.g3 * x.g8 * x.g8 - T(11) * x.g4 * x.g8 * x.g8 - T(11) * x.g5 * x.g8 * x.g8 - T(11) * x.g6 * x.g8 * x.g8 + T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9) + (T(16) * x.g2 * x.g9 - T(44) * x.g1 * x.g2 * x.g9 - T(20) * x.g2 * x.g2 * x.g9 - T(48) * x.g1 * x.g3 * x.g9 - T(28) * x.g2 * x.g3 * x.g9 + T(16) * x.g4 * x.g9) + (-T(44) * x.g1 * x.g4 * x.g9 - T(48) * x.g2 * x.g4 * x.g9 - T(48) * x.g3 * x.g4 * x.g9 - T(20) * x.g4 * x.g4 * x.g9 + T(12) * x.g5 * x.g9 - T(48) * x.g1 * x.g5 * x.g9) + (-T(40) * x.g2 * x.g5 * x.g9 - T(28) * x.g3 * x.g5 * x.g9 - T(40) * x.g4 * x.g5 * x.g9 - T(16) * x.g5 * x.g5 * x.g9 - T(44) * x.g1 * x.g6 * x.g9 - T(24) * x.g2 * x.g6 * x.g9) + (-T(36) * x.g4 * x.g6 * x.g9 - T(20) * x.g5 * x.g6 * x.g9 - T(48) * x.g1 * x.g7 * x.g9 - T(48) * x.g2 * x.g7 * x.g9 - T(48) * x.g3 * x.g7 * x.g9 - T(28) * x.g4 * x.g7 * x.g9) + (-T(28) * x.g5 * x.g7 * x.g9 - T(28) * x.g6 * x.g7 * x.g9 - T(44) * x.g1 * x.g8 * x.g9 - T(36) * x.g2 * x.g8 * x.g9 - T(28) * x.g3 * x.g8 * x.g9 - T(24) * x.g4 * x.g8 * x.g9) + (-T(20) * x.g5 * x.g8 * x.g9 - T(16) * x.g6 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(8) * x.g2 * x.g9 * x.g9 - T(8) * x.g4 * x.g9 * x.g9 - T(4) * x.g5 * x.g9 * x.g9) ) * T(0.0625)) * x.w4;
}
template <typename T>
LDK_DEV void geno_stats_P3(const GenoFeat<T>* f, T* acc) {
    const T v0 = f[0].DD1;  // dd1(0,)
    const T v1 = T(4) * (f[0].D * f[1].D) * (f[0].r2 * f[1].r2);  // dd2(0, 1)
    const T v2 = T(4) * (f[0].D * f[2].D) * (f[0].r2 * f[2].r2);  // dd2(0, 2)
    const T v3 = f[1].DD1;  // dd1(1,)
    const T v4 = T(4) * (f[1].D * f[2].D) * (f[1].r2 * f[2].r2);  // dd2(1, 2)
    const T v5 = f[2].DD1;  // dd1(2,)
    const T v6 = f[0].DZ1;  // dz_iii(0,)
    const T v7 = (T(2) * f[0].U * f[1].A) * (f[0].u3 * f[1].u1);  // dz_iij(0, 1)
    const T v8 = (T(2) * f[0].V * f[1].Bv) * (f[0].u3 * f[1].u1);  // dz_iji(0, 1)
    const T v9 = (T(2) * f[0].U * f[2].A) * (f[0].u3 * f[2].u1);  // dz_iij(0, 2)
    const T v10 = (T(2) * f[0].V * f[2].Bv) * (f[0].u3 * f[2].u1);  // dz_iji(0, 2)
    const T v11 = (T(2) * f[0].D * f[1].Wjj) * (f[1].u2 * f[0].u2);  // dz_ijj(0, 1)
    const T v12 = (T(2) * f[0].D * f[1].Bv * f[2].A) * (f[0].u2 * f[1].u1 * f[2].u1);  // dz_ijk(0, 1, 2)
    const T v13 = (T(2) * f[0].D * f[2].Bv * f[1].A) * (f[0].u2 * f[2].u1 * f[1].u1);  // dz_ijk(0, 2, 1)
    const T v14 = (T(2) * f[0].D * f[2].Wjj) * (f[2].u2 * f[0].u2);  // dz_ijj(0, 2)
    const T v15 = (T(2) * f[1].D * f[0].Wjj) * (f[0].u2 * f[1].u2);  // dz_ijj(1, 0)
    const T v16 = (T(2) * f[1].V * f[0].Bv) * (f[1].u3 * f[0].u1);  // dz_iji(1, 0)
    const T v17 = (T(2) * f[1].U * f[0].A) * (f[1].u3 * f[0].u1);  // dz_iij(1, 0)
    const T v18 = (T(2) * f[1].D * f[0].Bv * f[2].A) * (f[1].u2 * f[0].u1 * f[2].u1);  // dz_ijk(1, 0, 2)
    const T v19 = (T(2) * f[1].D * f[2].Bv * f[0].A) * (f[1].u2 * f[2].u1 * f[0].u1);  // dz_ijk(1, 2, 0)
    const T v20 = f[1].DZ1;  // dz_iii(1,)
    const T v21 = (T(2) * f[1].U * f[2].A) * (f[1].u3 * f[2].u1);  // dz_iij(1, 2)
    const T v22 = (T(2) * f[1].V * f[2].Bv) * (f[1].u3 * f[2].u1);  // dz_iji(1, 2)
    const T v23 = (T(2) * f[1].D * f[2].Wjj) * (f[2].u2 * f[1].u2);  // dz_ijj(1, 2)
    const T v24 = (T(2) * f[2].D * f[0].Wjj) * (f[0].u2 * f[2].u2);  // dz_ijj(2, 0)
    const T v25 = (T(2) * f[2].D * f[0].Bv * f[1].A) * (f[2].u2 * f[0].u1 * f[1].u1);  // dz_ijk(2, 0, 1)
    const T v26 = (T(2) * f[2].D * f[1].Bv * f[0].A) * (f[2].u2 * f[1].u1 * f[0].u1);  // dz_ijk(2, 1, 0)
    const T v27 = (T(2) * f[2].V * f[0].Bv) * (f[2].u3 * f[0].u1);  // dz_iji(2, 0)
    const T v28 = (T(2) * f[2].U * f[0].A) * (f[2].u3 * f[0].u1);  // dz_iij(2, 0)
    const T v29 = (T(2) * f[2].D * f[1].Wjj) * (f[1].u2 * f[2].u2);  // dz_ijj(2, 1)
    const T v30 = (T(2) * f[2].V * f[1].Bv) * (f[2].u3 * f[1].u1);  // dz_iji(2, 1)
    const T v31 = (T(2) * f[2].U * f[1].A) * (f[2].u3 * f[1].u1);  // dz_iij(2, 1)
    const T v32 = f[2].DZ1;  // dz_iii(2,)
    const T v33 = f[0].PI1;  // pi2_same(0,)
    const T v34 = (f[0].AQ3 * f[1].pB + f[0].AS3 * f[1].qB) * (f[0].r3 * f[1].r1);  // pi2_iiij(0, 1)
    const T v35 = (f[0].BP3 * f[1].pA + f[0].BR3 * f[1].qA) * (f[0].r3 * f[1].r1);  // pi2_ijii(0, 1)
    const T v36 = (f[0].AQ3 * f[2].pB + f[0].AS3 * f[2].qB) * (f[0].r3 * f[2].r1);  // pi2_iiij(0, 2)
    const T v37 = (f[0].BP3 * f[2].pA + f[0].BR3 * f[2].qA) * (f[0].r3 * f[2].r1);  // pi2_ijii(0, 2)
    const T v38 = f[0].BL * f[1].BR;  // pi2_iikk(0, 1)
    const T v39 = f[1].BL * f[0].BR;  // pi2_iikk(1, 0)
    const T v40 = f[0].BL * T(0.5) * (f[1].q * f[2].s + f[1].s * f[2].q);  // pi2_iikl(0, 1, 2)
    const T v41 = T(0.5) * (f[1].p * f[2].r + f[1].r * f[2].p) * f[0].BR;  // pi2_ijkk(1, 2, 0)
    const T v42 = f[0].BL * f[2].BR;  // pi2_iikk(0, 2)
    const T v43 = f[2].BL * f[0].BR;  // pi2_iikk(2, 0)
    const T v44 = (-T(0.25) * (f[0].qA * f[0].qB) * f[1].pB - T(0.25) * f[0].xab * (f[1].pA * f[1].pB) + T(0.25) * (f[0].qA * f[0].qB) * (f[1].pA * f[1].pB) - T(0.25) * f[0].qA * (f[1].pA * f[1].qB) - T(0.25) * (f[0].pA * f[0].pB) * f[1].xab - T(0.25) * (f[0].qA * f[0].qB) * f[1].xab + T(0.25) * (f[0].pA * f[0].qB) * f[1].xab + T(0.25) * (f[0].pB * f[0].qA) * f[1].xab - T(0.25) * (f[0].pA * f[0].qA) * f[1].qB + T(0.25) * (f[0].qA * (T(1) + f[0].xAb - f[0].xaB)) * f[1].qB + T(0.25) * f[0].xab * (f[1].pA * f[1].qB) + T(0.25) * (f[0].pB * f[0].qA) * (f[1].pA * f[1].qB) + T(0.25) * (f[0].qB * (T(1) + f[0].qA)) * f[1].qA - T(0.25) * f[0].xAb * (f[1].pB * f[1].qA) + T(0.25) * (f[0].pA * f[0].qB) * (f[1].pB * f[1].qA) - T(0.25) * (f[0].pA * f[0].qB) * f[1].qA - T(0.25) * f[0].pA * (f[1].qA * f[1].qB) + T(0.25) * f[0].xAb * (f[1].qA * f[1].qB) + T(0.25) * (f[0].pA * f[0].pB) * (f[1].qA * f[1].qB) + T(0.25) * f[0].xab * f[1].Bsgn + T(0.25) * f[0].Bsgn * f[1].xab - f[0].xab * f[1].xab) * (f[0].r2 * f[1].r2);  // pi2_ijij(0, 1)
    const T v45 = (-T(0.25) * (f[1].qA * f[1].qB) * f[0].pB - T(0.25) * f[1].xab * (f[0].pA * f[0].pB) + T(0.25) * (f[1].qA * f[1].qB) * (f[0].pA * f[0].pB) - T(0.25) * f[1].qA * (f[0].pA * f[0].qB) - T(0.25) * (f[1].pA * f[1].pB) * f[0].xab - T(0.25) * (f[1].qA * f[1].qB) * f[0].xab + T(0.25) * (f[1].pA * f[1].qB) * f[0].xab + T(0.25) * (f[1].pB * f[1].qA) * f[0].xab - T(0.25) * (f[1].pA * f[1].qA) * f[0].qB + T(0.25) * (f[1].qA * (T(1) + f[1].xAb - f[1].xaB)) * f[0].qB + T(0.25) * f[1].xab * (f[0].pA * f[0].qB) + T(0.25) * (f[1].pB * f[1].qA) * (f[0].pA * f[0].qB) + T(0.25) * (f[1].qB * (T(1) + f[1].qA)) * f[0].qA - T(0.25) * f[1].xAb * (f[0].pB * f[0].qA) + T(0.25) * (f[1].pA * f[1].qB) * (f[0].pB * f[0].qA) - T(0.25) * (f[1].pA * f[1].qB) * f[0].qA - T(0.25) * f[1].pA * (f[0].qA * f[0].qB) + T(0.25) * f[1].xAb * (f[0].qA * f[0].qB) + T(0.25) * (f[1].pA * f[1].pB) * (f[0].qA * f[0].qB) + T(0.25) * f[1].xab * f[0].Bsgn + T(0.25) * f[1].Bsgn * f[0].xab - f[1].xab * f[0].xab) * (f[1].r2 * f[0].r2);  // pi2_ijij(1, 0)
    const T v46 = f[1].r * (f[0].C00 * f[2].s + f[0].C01 * f[2].q) + f[1].p * (f[0].C10 * f[2].s + f[0].C11 * f[2].q);  // pi2_shared(0, 1, 2)
    const T v47 = f[2].r * (f[0].C00 * f[1].s + f[0].C01 * f[1].q) + f[2].p * (f[0].C10 * f[1].s + f[0].C11 * f[1].q);  // pi2_shared(0, 2, 1)
    const T v48 = (f[1].BP3 * f[0].pA + f[1].BR3 * f[0].qA) * (f[1].r3 * f[0].r1);  // pi2_ijii(1, 0)
    const T v49 = (f[1].AQ3 * f[0].pB + f[1].AS3 * f[0].qB) * (f[1].r3 * f[0].r1);  // pi2_iiij(1, 0)
    const T v50 = f[0].r * (f[1].C00 * f[2].s + f[1].C01 * f[2].q) + f[0].p * (f[1].C10 * f[2].s + f[1].C11 * f[2].q);  // pi2_shared(1, 0, 2)
    const T v51 = f[2].r * (f[1].C00 * f[0].s + f[1].C01 * f[0].q) + f[2].p * (f[1].C10 * f[0].s + f[1].C11 * f[0].q);  // pi2_shared(1, 2, 0)
    const T v52 = T(0.5) * (f[0].p * f[1].r + f[0].r * f[1].p) * f[2].BR;  // pi2_ijkk(0, 1, 2)
    const T v53 = f[2].BL * T(0.5) * (f[0].q * f[1].s + f[0].s * f[1].q);  // pi2_iikl(2, 0, 1)
    const T v54 = (-T(0.25) * (f[0].qA * f[0].qB) * f[2].pB - T(0.25) * f[0].xab * (f[2].pA * f[2].pB) + T(0.25) * (f[0].qA * f[0].qB) * (f[2].pA * f[2].pB) - T(0.25) * f[0].qA * (f[2].pA * f[2].qB) - T(0.25) * (f[0].pA * f[0].pB) * f[2].xab - T(0.25) * (f[0].qA * f[0].qB) * f[2].xab + T(0.25) * (f[0].pA * f[0].qB) * f[2].xab + T(0.25) * (f[0].pB * f[0].qA) * f[2].xab - T(0.25) * (f[0].pA * f[0].qA) * f[2].qB + T(0.25) * (f[0].qA * (T(1) + f[0].xAb - f[0].xaB)) * f[2].qB + T(0.25) * f[0].xab * (f[2].pA * f[2].qB) + T(0.25) * (f[0].pB * f[0].qA) * (f[2].pA * f[2].qB) + T(0.25) * (f[0].qB * (T(1) + f[0].qA)) * f[2].qA - T(0.25) * f[0].xAb * (f[2].pB * f[2].qA) + T(0.25) * (f[0].pA * f[0].qB) * (f[2].pB * f[2].qA) - T(0.25) * (f[0].pA * f[0].qB) * f[2].qA - T(0.25) * f[0].pA * (f[2].qA * f[2].qB) + T(0.25) * f[0].xAb * (f[2].qA * f[2].qB) + T(0.25) * (f[0].pA * f[0].pB) * (f[2].qA * f[2].qB) + T(0.25) * f[0].xab * f[2].Bsgn + T(0.25) * f[0].Bsgn * f[2].xab - f[0].xab * f[2].xab) * (f[0].r2 * f[2].r2);  // pi2_ijij(0, 2)
    const T v55 = (-T(0.25) * (f[2].qA * f[2].qB) * f[0].pB - T(0.25) * f[2].xab * (f[0].pA * f[0].pB) + T(0.25) * (f[2].qA * f[2].qB) * (f[0].pA * f[0].pB) - T(0.25) * f[2].qA * (f[0].pA * f[0].qB) - T(0.25) * (f[2].pA * f[2].pB) * f[0].xab - T(0.25) * (f[2].qA * f[2].qB) * f[0].xab + T(0.25) * (f[2].pA * f[2].qB) * f[0].xab + T(0.25) * (f[2].pB * f[2].qA) * f[0].xab - T(0.25) * (f[2].pA * f[2].qA) * f[0].qB + T(0.25) * (f[2].qA * (T(1) + f[2].xAb - f[2].xaB)) * f[0].qB + T(0.25) * f[2].xab * (f[0].pA * f[0].qB) + T(0.25) * (f[2].pB * f[2].qA) * (f[0].pA * f[0].qB) + T(0.25) * (f[2].qB * (T(1) + f[2].qA)) * f[0].qA - T(0.25) * f[2].xAb * (f[0].pB * f[0].qA) + T(0.25) * (f[2].pA * f[2].qB) * (f[0].pB * f[0].qA) - T(0.25) * (f[2].pA * f[2].qB) * f[0].qA - T(0.25) * f[2].pA * (f[0].qA * f[0].qB) + T(0.25) * f[2].xAb * (f[0].qA * f[0].qB) + T(0.25) * (f[2].pA * f[2].pB) * (f[0].qA * f[0].qB) + T(0.25) * f[2].xab * f[0].Bsgn + T(0.25) * f[2].Bsgn * f[0].xab - f[2].xab * f[0].xab) * (f[2].r2 * f[0].r2);  // pi2_ijij(2, 0)
    const T v56 = T(0.5) * (f[0].p * f[2].r + f[0].r * f[2].p) * f[1].BR;  // pi2_ijkk(0, 2, 1)
    const T v57 = f[1].BL * T(0.5) * (f[0].q * f[2].s + f[0].s * f[2].q);  // pi2_iikl(1, 0, 2)
    const T v58 = f[0].r * (f[2].C00 * f[1].s + f[2].C01 * f[1].q) + f[0].p * (f[2].C10 * f[1].s + f[2].C11 * f[1].q);  // pi2_shared(2, 0, 1)
    const T v59 = f[1].r * (f[2].C00 * f[0].s + f[2].C01 * f[0].q) + f[1].p * (f[2].C10 * f[0].s + f[2].C11 * f[0].q);  // pi2_shared(2, 1, 0)
    const T v60 = (f[2].BP3 * f[0].pA + f[2].BR3 * f[0].qA) * (f[2].r3 * f[0].r1);  // pi2_ijii(2, 0)
    const T v61 = (f[2].AQ3 * f[0].pB + f[2].AS3 * f[0].qB) * (f[2].r3 * f[0].r1);  // pi2_iiij(2, 0)
    const T v62 = f[1].PI1;  // pi2_same(1,)
    const T v63 = (f[1].AQ3 * f[2].pB + f[1].AS3 * f[2].qB) * (f[1].r3 * f[2].r1);  // pi2_iiij(1, 2)
    const T v64 = (f[1].BP3 * f[2].pA + f[1].BR3 * f[2].qA) * (f[1].r3 * f[2].r1);  // pi2_ijii(1, 2)
    const T v65 = f[1].BL * f[2].BR;  // pi2_iikk(1, 2)
    const T v66 = f[2].BL * f[1].BR;  // pi2_iikk(2, 1)
    const T v67 = (-T(0.25) * (f[1].qA * f[1].qB) * f[2].pB - T(0.25) * f[1].xab * (f[2].pA * f[2].pB) + T(0.25) * (f[1].qA * f[1].qB) * (f[2].pA * f[2].pB) - T(0.25) * f[1].qA * (f[2].pA * f[2].qB) - T(0.25) * (f[1].pA * f[1].pB) * f[2].xab - T(0.25) * (f[1].qA * f[1].qB) * f[2].xab + T(0.25) * (f[1].pA * f[1].qB) * f[2].xab + T(0.25) * (f[1].pB * f[1].qA) * f[2].xab - T(0.25) * (f[1].pA * f[1].qA) * f[2].qB + T(0.25) * (f[1].qA * (T(1) + f[1].xAb - f[1].xaB)) * f[2].qB + T(0.25) * f[1].xab * (f[2].pA * f[2].qB) + T(0.25) * (f[1].pB * f[1].qA) * (f[2].pA * f[2].qB) + T(0.25) * (f[1].qB * (T(1) + f[1].qA)) * f[2].qA - T(0.25) * f[1].xAb * (f[2].pB * f[2].qA) + T(0.25) * (f[1].pA * f[1].qB) * (f[2].pB * f[2].qA) - T(0.25) * (f[1].pA * f[1].qB) * f[2].qA - T(0.25) * f[1].pA * (f[2].qA * f[2].qB) + T(0.25) * f[1].xAb * (f[2].qA * f[2].qB) + T(0.25) * (f[1].pA * f[1].pB) * (f[2].qA * f[2].qB) + T(0.25) * f[1].xab * f[2].Bsgn + T(0.25) * f[1].Bsgn * f[2].xab - f[1].xab * f[2].xab) * (f[1].r2 * f[2].r2);  // pi2_ijij(1, 2)
    const T v68 = (-T(0.25) * (f[2].qA * f[2].qB) * f[1].pB - T(0.25) * f[2].xab * (f[1].pA * f[1].pB) + T(0.25) * (f[2].qA * f[2].qB) * (f[1].pA * f[1].pB) - T(0.25) * f[2].qA * (f[1].pA * f[1].qB) - T(0.25) * (f[2].pA * f[2].pB) * f[1].xab - T(0.25) * (f[2].qA * f[2].qB) * f[1].xab + T(0.25) * (f[2].pA * f[2].qB) * f[1].xab + T(0.25) * (f[2].pB * f[2].qA) * f[1].xab - T(0.25) * (f[2].pA * f[2].qA) * f[1].qB + T(0.25) * (f[2].qA * (T(1) + f[2].xAb - f[2].xaB)) * f[1].qB + T(0.25) * f[2].xab * (f[1].pA * f[1].qB) + T(0.25) * (f[2].pB * f[2].qA) * (f[1].pA * f[1].qB) + T(0.25) * (f[2].qB * (T(1) + f[2].qA)) * f[1].qA - T(0.25) * f[2].xAb * (f[1].pB * f[1].qA) + T(0.25) * (f[2].pA * f[2].qB) * (f[1].pB * f[1].qA) - T(0.25) * (f[2].pA * f[2].qB) * f[1].qA - T(0.25) * f[2].pA * (f[1].qA * f[1].qB) + T(0.25) * f[2].xAb * (f[1].qA * f[1].qB) + T(0.25) * (f[2].pA * f[2].pB) * (f[1].qA * f[1].qB) + T(0.25) * f[2].xab * f[1].Bsgn + T(0.25) * f[2].Bsgn * f[1].xab - f[2].xab * f[1].xab) * (f[2].r2 * f[1].r2);  // pi2_ijij(2, 1)
    const T v69 = (f[2].BP3 * f[1].pA + f[2].BR3 * f[1].qA) * (f[2].r3 * f[1].r1);  // pi2_ijii(2, 1)
    const T v70 = (f[2].AQ3 * f[1].pB + f[2].AS3 * f[1].qB) * (f[2].r3 * f[1].r1);  // pi2_iiij(2, 1)
    const T v71 = f[2].PI1;  // pi2_same(2,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // DD_0_1
    acc[2] += v2;  // DD_0_2
    acc[3] += v3;  // DD_1_1
    acc[4] += v4;  // DD_1_2
    acc[5] += v5;  // DD_2_2
    acc[6] += v6;  // Dz_0_0_0
    acc[7] += T(0.5) * (v7 + v8);  // Dz_0_0_1
    acc[8] += T(0.5) * (v9 + v10);  // Dz_0_0_2
    acc[9] += v11;  // Dz_0_1_1
    acc[10] += T(0.5) * (v12 + v13);  // Dz_0_1_2
    acc[11] += v14;  // Dz_0_2_2
    acc[12] += v15;  // Dz_1_0_0
    acc[13] += T(0.5) * (v16 + v17);  // Dz_1_0_1
    acc[14] += T(0.5) * (v18 + v19);  // Dz_1_0_2
    acc[15] += v20;  // Dz_1_1_1
    acc[16] += T(0.5) * (v21 + v22);  // Dz_1_1_2
    acc[17] += v23;  // Dz_1_2_2
    acc[18] += v24;  // Dz_2_0_0
    acc[19] += T(0.5) * (v25 + v26);  // Dz_2_0_1
    acc[20] += T(0.5) * (v27 + v28);  // Dz_2_0_2
    acc[21] += v29;  // Dz_2_1_1
    acc[22] += T(0.5) * (v30 + v31);  // Dz_2_1_2
    acc[23] += v32;  // Dz_2_2_2
    acc[24] += v33;  // pi2_0_0_0_0
    acc[25] += T(0.5) * (v34 + v35);  // pi2_0_0_0_1
    acc[26] += T(0.5) * (v36 + v37);  // pi2_0_0_0_2
    acc[27] += T(0.5) * (v38 + v39);  // pi2_0_0_1_1
    acc[28] += T(0.5) * (v40 + v41);  // pi2_0_0_1_2
    acc[29] += T(0.5) * (v42 + v43);  // pi2_0_0_2_2
    acc[30] += T(0.5) * (v44 + v45);  // pi2_0_1_0_1
    acc[31] += T(0.5) * (v46 + v47);  // pi2_0_1_0_2
    acc[32] += T(0.5) * (v48 + v49);  // pi2_0_1_1_1
    acc[33] += T(0.5) * (v50 + v51);  // pi2_0_1_1_2
    acc[34] += T(0.5) * (v52 + v53);  // pi2_0_1_2_2
    acc[35] += T(0.5) * (v54 + v55);  // pi2_0_2_0_2
    acc[36] += T(0.5) * (v56 + v57);  // pi2_0_2_1_1
    acc[37] += T(0.5) * (v58 + v59);  // pi2_0_2_1_2
    acc[38] += T(0.5) * (v60 + v61);  // pi2_0_2_2_2
    acc[39] += v62;  // pi2_1_1_1_1
    acc[40] += T(0.5) * (v63 + v64);  // pi2_1_1_1_2
    acc[41] += T(0.5) * (v65 + v66);  // pi2_1_1_2_2
    acc[42] += T(0.5) * (v67 + v68);  // pi2_1_2_1_2
    acc[43] += T(0.5) * (v69 + v70);  // pi2_1_2_2_2
    acc[44] += v71;  // pi2_2_2_2_2
}

// genotype path, P = 4: 105 statistics from 180 distinct raw calls
template <typename T>
LDK_DEV void geno_features_P4(GenoFeat<T>& x) {
    geno_prepare(x);
    x.xAB = x.g1 + T(0.5) * x.g2 + T(0.5) * x.g4 + T(0.25) * x.g5;
    x.xAb = T(0.5) * x.g2 + x.g3 + T(0.25) * x.g5 + T(0.5) * x.g6;
    x.xaB = T(0.5) * x.g4 + T(0.25) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.xab = T(0.25) * x.g5 + T(0.5) * x.g6 + T(0.5) * x.g8 + x.g9;
    x.D = x.xAB * x.xab - x.xAb * x.xaB;
    x.pA = x.g1 + x.g2 + x.g3 + T(0.5) * (x.g4 + x.g5 + x.g6);
    x.qA = T(0.5) * (x.g4 + x.g5 + x.g6) + x.g7 + x.g8 + x.g9;
    x.pB = x.g1 + T(0.5) * x.g2 + x.g4 + T(0.5) * x.g5 + x.g7 + T(0.5) * x.g8;
    x.qB = T(0.5) * x.g2 + x.g3 + T(0.5) * x.g5 + x.g6 + T(0.5) * x.g8 + x.g9;
    x.BL = (T(4) * x.pA * x.qA - (x.g4 + x.g5 + x.g6)) * x.inn1;
    x.BR = (T(4) * x.pB * x.qB - (x.g2 + x.g5 + x.g8)) * x.inn1;
    x.C00 = (x.pA * x.pB - x.xAB) * x.inn1;
    x.C01 = (x.pA * x.qB - x.xAb) * x.inn1;
    x.C10 = (x.qA * x.pB - x.xaB) * x.inn1;
    x.C11 = (x.qA * x.qB - x.xab) * x.inn1;
    x.Bsgn = x.xAB - x.xAb - x.xaB + x.xab;
    x.p = x.pA * x.invn;
    x.r = x.qA * x.invn;
    x.q = x.pB * x.invn;
    x.s = x.qB * x.invn;
    x.L0 = x.g5 + T(2) * x.g6 + T(2) * x.g8 + T(4) * x.g9;
    x.AQ3 = -(x.qB * (T(3) * x.g4 + T(3) * x.g5 + T(3) * x.g6 + T(4) * x.g7 + T(4) * x.g8 + T(4) * x.g9)) / T(8) + x.pA * x.qB * x.qA / T(2) + (x.qA * x.L0) / T(8) + (x.g5 + T(2) * x.g6) / T(8) - (x.pA * x.L0) / T(8);
    x.AS3 = -(x.pB * (T(5) * x.g4 + T(5) * x.g5 + T(5) * x.g6 + T(8) * x.g7 + T(8) * x.g8 + T(8) * x.g9)) / T(8) + x.pA * x.pB * x.qA / T(2) + (x.qA * (-T(2) * x.g2 - T(4) * x.g3 + T(4) * x.g4 + x.g5 - T(2) * x.g6 + T(8) * x.g7 + T(4) * x.g8 + T(4))) / T(8) + (-x.g5 - T(2) * x.g6 - T(4) * x.g7 - T(4) * x.g8 - T(4) * x.g9) / T(8) + (x.pA * x.L0) / T(8);
    x.BP3 = -(x.qA * (T(3) * x.g2 + T(4) * x.g3 + T(3) * x.g5 + T(4) * x.g6 + T(3) * x.g8 + T(4) * x.g9)) / T(8) + x.pB * x.qB * x.qA / T(2) + (x.qB * x.L0) / T(8) + (x.g5 + T(2) * x.g8) / T(8) - (x.pB * x.L0) / T(8);
    x.BR3 = -(x.pA * (T(5) * x.g2 + T(8) * x.g3 + T(5) * x.g5 + T(8) * x.g6 + T(5) * x.g8 + T(8) * x.g9)) / T(8) + x.pA * x.pB * x.qB / T(2) + (x.qB * (T(4) * x.g2 + T(8) * x.g3 - T(2) * x.g4 + x.g5 + T(4) * x.g6 - T(4) * x.g7 - T(2) * x.g8 + T(4))) / T(8) + (-T(4) * x.g3 - x.g5 - T(4) * x.g6 - T(2) * x.g8 - T(4) * x.g9) / T(8) + (x.pB * x.L0) / T(8);
    x.A = -x.g1 + x.g3 - x.g4 + x.g6 - x.g7 + x.g9;
    x.Bv = -x.g1 - x.g2 - x.g3 + x.g7 + x.g8 + x.g9;
    x.Wjj = (-x.g1 + x.g3 + x.g7 - x.g9) + x.A * x.Bv;
    x.U = x.D * (T(1) + x.Bv) + T(0.25) * (T(2) * x.g2 * x.g7 + T(4) * x.g3 * x.g7 + T(2) * x.g5 * x.g7 + T(4) * x.g6 * x.g7 - T(2) * x.g1 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g4 * x.g8 + T(2) * x.g6 * x.g8 - T(4) * x.g1 * x.g9 - T(2) * x.g2 * x.g9 - T(4) * x.g4 * x.g9 - T(2) * x.g5 * x.g9);
    x.V = x.D * (T(1) + x.A) + T(0.25) * (T(2) * x.g3 * x.g4 + T(2) * x.g3 * x.g5 - T(2) * x.g1 * x.g6 - T(2) * x.g2 * x.g6 + T(4) * x.g3 * x.g7 + T(2) * x.g6 * x.g7 + T(4) * x.g3 * x.g8 + T(2) * x.g6 * x.g8 - T(4) * x.g1 * x.g9 - T(4) * x.g2 * x.g9 - T(2) * x.g4 * x.g9 - T(2) * x.g5 * x.g9);
    x.DD1 = T(4) * (((x.g2 * x.g4 - x.g2 * x.g2 * x.g4 + T(4) * x.g3 * x.g4 - T(4) * x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4) + (-x.g2 * x.g4 * x.g4 - T(4) * x.g3 * x.g4 * x.g4) + (x.g1 * x.g5 - x.g1 * x.g1 * x.g5 + x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g3 * x.g3 * x.g5 - T(4) * x.g3 * x.g4 * x.g5 - x.g1 * x.g5 * x.g5 - x.g3 * x.g5 * x.g5) + (T(4) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 + x.g2 * x.g6 - T(4) * x.g1 * x.g2 * x.g6 - x.g2 * x.g2 * x.g6 + T(2) * x.g2 * x.g4 * x.g6 - T(4) * x.g1 * x.g5 * x.g6 - T(4) * x.g1 * x.g6 * x.g6 - x.g2 * x.g6 * x.g6) + (T(4) * x.g2 * x.g7 - T(4) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7 - T(16) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(4) * x.g2 * x.g4 * x.g7 - T(16) * x.g3 * x.g4 * x.g7 + x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 - T(4) * x.g2 * x.g5 * x.g7 - T(18) * x.g3 * x.g5 * x.g7 - x.g5 * x.g5 * x.g7 + T(4) * x.g6 * x.g7 + T(8) * x.g1 * x.g6 * x.g7 - T(16) * x.g3 * x.g6 * x.g7 - T(4) * x.g5 * x.g6 * x.g7 - T(4) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7) + (T(4) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 + T(4) * x.g3 * x.g8 + T(8) * x.g1 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 + x.g4 * x.g8 - T(4) * x.g1 * x.g4 * x.g8 + T(2) * x.g2 * x.g4 * x.g8 - x.g4 * x.g4 * x.g8 - T(4) * x.g1 * x.g5 * x.g8 - T(4) * x.g3 * x.g5 * x.g8 + x.g6 * x.g8 + T(2) * x.g2 * x.g6 * x.g8 - T(4) * x.g3 * x.g6 * x.g8 + T(2) * x.g4 * x.g6 * x.g8 - x.g6 * x.g6 * x.g8 - T(16) * x.g3 * x.g7 * x.g8 - T(4) * x.g6 * x.g7 * x.g8 - T(4) * x.g1 * x.g8 * x.g8 - T(4) * x.g3 * x.g8 * x.g8 - x.g4 * x.g8 * x.g8 - x.g6 * x.g8 * x.g8) + (T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9 + T(4) * x.g2 * x.g9 - T(16) * x.g1 * x.g2 * x.g9 - T(4) * x.g2 * x.g2 * x.g9 + T(4) * x.g4 * x.g9 - T(16) * x.g1 * x.g4 * x.g9 + T(8) * x.g3 * x.g4 * x.g9 - T(4) * x.g4 * x.g4 * x.g9 + x.g5 * x.g9 - T(18) * x.g1 * x.g5 * x.g9 - T(4) * x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 - T(4) * x.g4 * x.g5 * x.g9 - x.g5 * x.g5 * x.g9 - T(16) * x.g1 * x.g6 * x.g9 - T(4) * x.g2 * x.g6 * x.g9 + T(8) * x.g2 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 - T(16) * x.g1 * x.g8 * x.g9 - T(4) * x.g4 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - x.g5 * x.g9 * x.g9) ) * T(0.0625) + x.D * x.D) * x.w4;
    x.DZ1 = T(2) * (T(0.25) * (-(x.g2 * x.g4) + T(3) * x.g1 * x.g2 * x.g4 + x.g2 * x.g2 * x.g4 + T(2) * x.g3 * x.g4 + T(4) * x.g1 * x.g3 * x.g4 - x.g2 * x.g3 * x.g4 - T(4) * x.g3 * x.g3 * x.g4 + x.g2 * x.g4 * x.g4 + T(2) * x.g3 * x.g4 * x.g4 + T(2) * x.g1 * x.g5 - T(3) * x.g1 * x.g1 * x.g5 - x.g1 * x.g2 * x.g5 + T(2) * x.g3 * x.g5 + T(2) * x.g1 * x.g3 * x.g5 - x.g2 * x.g3 * x.g5 - T(3) * x.g3 * x.g3 * x.g5 - x.g1 * x.g4 * x.g5 + x.g3 * x.g4 * x.g5 + T(2) * x.g1 * x.g6 - T(4) * x.g1 * x.g1 * x.g6 - x.g2 * x.g6 - x.g1 * x.g2 * x.g6 + x.g2 * x.g2 * x.g6 + T(4) * x.g1 * x.g3 * x.g6 + T(3) * x.g2 * x.g3 * x.g6 - T(2) * x.g1 * x.g4 * x.g6 - T(2) * x.g2 * x.g4 * x.g6 - T(2) * x.g3 * x.g4 * x.g6 + x.g1 * x.g5 * x.g6 - x.g3 * x.g5 * x.g6 + T(2) * x.g1 * x.g6 * x.g6 + x.g2 * x.g6 * x.g6 + T(2) * x.g2 * x.g7 + T(4) * x.g1 * x.g2 * x.g7 + T(2) * x.g2 * x.g2 * x.g7 + T(8) * x.g3 * x.g7 + T(4) * x.g1 * x.g3 * x.g7 - T(4) * x.g3 * x.g3 * x.g7 - x.g2 * x.g4 * x.g7 + T(2) * x.g5 * x.g7 + T(2) * x.g1 * x.g5 * x.g7 + x.g2 * x.g5 * x.g7 + T(2) * x.g3 * x.g5 * x.g7 - x.g4 * x.g5 * x.g7 + T(2) * x.g6 * x.g7 - x.g2 * x.g6 * x.g7 - T(2) * x.g4 * x.g6 * x.g7 + x.g5 * x.g6 * x.g7 + T(2) * x.g6 * x.g6 * x.g7 - T(4) * x.g2 * x.g7 * x.g7 - T(4) * x.g3 * x.g7 * x.g7 - T(3) * x.g5 * x.g7 * x.g7 - T(4) * x.g6 * x.g7 * x.g7 + T(2) * x.g1 * x.g8 - T(4) * x.g1 * x.g1 * x.g8 - T(2) * x.g1 * x.g2 * x.g8 + T(2) * x.g3 * x.g8 - T(2) * x.g2 * x.g3 * x.g8 - T(4) * x.g3 * x.g3 * x.g8 - x.g4 * x.g8 - x.g1 * x.g4 * x.g8 - T(2) * x.g2 * x.g4 * x.g8 - x.g3 * x.g4 * x.g8 + x.g4 * x.g4 * x.g8 + x.g1 * x.g5 * x.g8 + x.g3 * x.g5 * x.g8 - x.g6 * x.g8 - x.g1 * x.g6 * x.g8 - T(2) * x.g2 * x.g6 * x.g8 - x.g3 * x.g6 * x.g8 - T(2) * x.g4 * x.g6 * x.g8 + x.g6 * x.g6 * x.g8 + T(4) * x.g1 * x.g7 * x.g8 - T(2) * x.g2 * x.g7 * x.g8 + T(3) * x.g4 * x.g7 * x.g8 - x.g5 * x.g7 * x.g8 - x.g6 * x.g7 * x.g8 + T(2) * x.g1 * x.g8 * x.g8 + T(2) * x.g3 * x.g8 * x.g8 + x.g4 * x.g8 * x.g8 + x.g6 * x.g8 * x.g8 + T(8) * x.g1 * x.g9 - T(4) * x.g1 * x.g1 * x.g9 + T(2) * x.g2 * x.g9 + T(2) * x.g2 * x.g2 * x.g9 + T(4) * x.g1 * x.g3 * x.g9 + T(4) * x.g2 * x.g3 * x.g9 + T(2) * x.g4 * x.g9 - x.g2 * x.g4 * x.g9 + T(2) * x.g4 * x.g4 * x.g9 + T(2) * x.g5 * x.g9 + T(2) * x.g1 * x.g5 * x.g9 + x.g2 * x.g5 * x.g9 + T(2) * x.g3 * x.g5 * x.g9 + x.g4 * x.g5 * x.g9 - x.g2 * x.g6 * x.g9 - T(2) * x.g4 * x.g6 * x.g9 - x.g5 * x.g6 * x.g9 + T(4) * x.g1 * x.g7 * x.g9 + T(4) * x.g3 * x.g7 * x.g9 + T(4) * x.g4 * x.g7 * x.g9 + T(2) * x.g5 * x.g7 * x.g9 + T(4) * x.g6 * x.g7 * x.g9 - T(2) * x.g2 * x.g8 * x.g9 + T(4) * x.g3 * x.g8 * x.g9 - x.g4 * x.g8 * x.g9 - x.g5 * x.g8 * x.g9 + T(3) * x.g6 * x.g8 * x.g9 - T(4) * x.g1 * x.g9 * x.g9 - T(4) * x.g2 * x.g9 * x.g9 - T(4) * x.g4 * x.g9 * x.g9 - T(3) * x.g5 * x.g9 * x.g9 ) + x.A * x.Bv * x.D) * x.w4;
    x.PI1 = (x.pA * x.pB * x.qB * x.qA + ((T(13) * x.g2 * x.g4 - T(16) * x.g1 * x.g2 * x.g4 - T(11) * x.g2 * x.g2 * x.g4 + T(16) * x.g3 * x.g4 - T(28) * x.g1 * x.g3 * x.g4 - T(24) * x.g2 * x.g3 * x.g4) + (-T(8) * x.g3 * x.g3 * x.g4 - T(11) * x.g2 * x.g4 * x.g4 - T(20) * x.g3 * x.g4 * x.g4 - T(6) * x.g5 + T(12) * x.g1 * x.g5 - T(4) * x.g1 * x.g1 * x.g5 + T(17) * x.g2 * x.g5) + (-T(20) * x.g1 * x.g2 * x.g5 - T(11) * x.g2 * x.g2 * x.g5 + T(12) * x.g3 * x.g5 - T(28) * x.g1 * x.g3 * x.g5 - T(20) * x.g2 * x.g3 * x.g5 - T(4) * x.g3 * x.g3 * x.g5) + (T(17) * x.g4 * x.g5 - T(20) * x.g1 * x.g4 * x.g5 - T(32) * x.g2 * x.g4 * x.g5 - T(40) * x.g3 * x.g4 * x.g5 - T(11) * x.g4 * x.g4 * x.g5 + T(11) * x.g5 * x.g5) + (-T(16) * x.g1 * x.g5 * x.g5 - T(17) * x.g2 * x.g5 * x.g5 - T(16) * x.g3 * x.g5 * x.g5 - T(17) * x.g4 * x.g5 * x.g5 - T(6) * x.g5 * x.g5 * x.g5 + T(16) * x.g1 * x.g6 - T(8) * x.g1 * x.g1 * x.g6) + (T(13) * x.g2 * x.g6 - T(24) * x.g1 * x.g2 * x.g6 - T(11) * x.g2 * x.g2 * x.g6 - T(28) * x.g1 * x.g3 * x.g6 - T(16) * x.g2 * x.g3 * x.g6 + T(24) * x.g4 * x.g6) + (-T(36) * x.g1 * x.g4 * x.g6 - T(38) * x.g2 * x.g4 * x.g6 - T(36) * x.g3 * x.g4 * x.g6 - T(20) * x.g4 * x.g4 * x.g6 + T(17) * x.g5 * x.g6 - T(40) * x.g1 * x.g5 * x.g6) + (-T(32) * x.g2 * x.g5 * x.g6 - T(20) * x.g3 * x.g5 * x.g6 - T(42) * x.g4 * x.g5 * x.g6 - T(17) * x.g5 * x.g5 * x.g6 - T(20) * x.g1 * x.g6 * x.g6 - T(11) * x.g2 * x.g6 * x.g6) + (-T(20) * x.g4 * x.g6 * x.g6 - T(11) * x.g5 * x.g6 * x.g6 + T(16) * x.g2 * x.g7 - T(28) * x.g1 * x.g2 * x.g7 - T(20) * x.g2 * x.g2 * x.g7 + T(16) * x.g3 * x.g7) + (-T(48) * x.g1 * x.g3 * x.g7 - T(44) * x.g2 * x.g3 * x.g7 - T(16) * x.g3 * x.g3 * x.g7 - T(24) * x.g2 * x.g4 * x.g7 - T(44) * x.g3 * x.g4 * x.g7) + (T(12) * x.g5 * x.g7 - T(28) * x.g1 * x.g5 * x.g7 - T(40) * x.g2 * x.g5 * x.g7 - T(48) * x.g3 * x.g5 * x.g7 - T(20) * x.g4 * x.g5 * x.g7 - T(16) * x.g5 * x.g5 * x.g7) + (T(16) * x.g6 * x.g7 - T(48) * x.g1 * x.g6 * x.g7 - T(48) * x.g2 * x.g6 * x.g7 - T(44) * x.g3 * x.g6 * x.g7 - T(36) * x.g4 * x.g6 * x.g7 - T(40) * x.g5 * x.g6 * x.g7) + (-T(20) * x.g6 * x.g6 * x.g7 - T(8) * x.g2 * x.g7 * x.g7 - T(16) * x.g3 * x.g7 * x.g7 - T(4) * x.g5 * x.g7 * x.g7 - T(8) * x.g6 * x.g7 * x.g7 + T(16) * x.g1 * x.g8 - T(8) * x.g1 * x.g1 * x.g8) + (T(24) * x.g2 * x.g8 - T(36) * x.g1 * x.g2 * x.g8 - T(20) * x.g2 * x.g2 * x.g8 + T(16) * x.g3 * x.g8 - T(48) * x.g1 * x.g3 * x.g8 - T(36) * x.g2 * x.g3 * x.g8 - T(8) * x.g3 * x.g3 * x.g8) + (T(13) * x.g4 * x.g8 - T(24) * x.g1 * x.g4 * x.g8 - T(38) * x.g2 * x.g4 * x.g8 - T(48) * x.g3 * x.g4 * x.g8 - T(11) * x.g4 * x.g4 * x.g8 + T(17) * x.g5 * x.g8 - T(40) * x.g1 * x.g5 * x.g8) + (-T(42) * x.g2 * x.g5 * x.g8 - T(40) * x.g3 * x.g5 * x.g8 - T(32) * x.g4 * x.g5 * x.g8 - T(17) * x.g5 * x.g5 * x.g8 + T(13) * x.g6 * x.g8 - T(48) * x.g1 * x.g6 * x.g8) + (-T(38) * x.g2 * x.g6 * x.g8 - T(24) * x.g3 * x.g6 * x.g8 - T(38) * x.g4 * x.g6 * x.g8 - T(32) * x.g5 * x.g6 * x.g8 - T(11) * x.g6 * x.g6 * x.g8 - T(28) * x.g1 * x.g7 * x.g8) + (-T(36) * x.g2 * x.g7 * x.g8 - T(44) * x.g3 * x.g7 * x.g8 - T(16) * x.g4 * x.g7 * x.g8 - T(20) * x.g5 * x.g7 * x.g8 - T(24) * x.g6 * x.g7 * x.g8 - T(20) * x.g1 * x.g8 * x.g8) + (-T(20) * x.g2 * x.g8 * x.g8 - T(20) * x.g3 * x.g8 * x.g8 - T(11) * x.g4 * x.g8 * x.g8 - T(11) * x.g5 * x.g8 * x.g8 - T(11) * x.g6 * x.g8 * x.g8 + T(16) * x.g1 * x.g9 - T(16) * x.g1 * x.g1 * x.g9) + (T(16) * x.g2 * x.g9 - T(44) * x.g1 * x.g2 * x.g9 - T(20) * x.g2 * x.g2 * x.g9 - T(48) * x.g1 * x.g3 * x.g9 - T(28) * x.g2 * x.g3 * x.g9 + T(16) * x.g4 * x.g9) + (-T(44) * x.g1 * x.g4 * x.g9 - T(48) * x.g2 * x.g4 * x.g9 - T(48) * x.g3 * x.g4 * x.g9 - T(20) * x.g4 * x.g4 * x.g9 + T(12) * x.g5 * x.g9 - T(48) * x.g1 * x.g5 * x.g9) + (-T(40) * x.g2 * x.g5 * x.g9 - T(28) * x.g3 * x.g5 * x.g9 - T(40) * x.g4 * x.g5 * x.g9 - T(16) * x.g5 * x.g5 * x.g9 - T(44) * x.g1 * x.g6 * x.g9 - T(24) * x.g2 * x.g6 * x.g9) + (-T(36) * x.g4 * x.g6 * x.g9 - T(20) * x.g5 * x.g6 * x.g9 - T(48) * x.g1 * x.g7 * x.g9 - T(48) * x.g2 * x.g7 * x.g9 - T(48) * x.g3 * x.g7 * x.g9 - T(28) * x.g4 * x.g7 * x.g9) + (-T(28) * x.g5 * x.g7 * x.g9 - T(28) * x.g6 * x.g7 * x.g9 - T(44) * x.g1 * x.g8 * x.g9 - T(36) * x.g2 * x.g8 * x.g9 - T(28) * x.g3 * x.g8 * x.g9 - T(24) * x.g4 * x.g8 * x.g9) + (-T(20) * x.g5 * x.g8 * x.g9 - T(16) * x.g6 * x.g8 * x.g9 - T(16) * x.g1 * x.g9 * x.g9 - T(8) * x.g2 * x.g9 * x.g9 - T(8) * x.g4 * x.g9 * x.g9 - T(4) * x.g5 * x.g9 * x.g9) ) * T(0.0625)) * x.w4;
}
template <typename T>
LDK_DEV void geno_stats_P4(const GenoFeat<T>* f, T* acc) {
    const T v0 = f[0].DD1;  // dd1(0,)
    const T v1 = T(4) * (f[0].D * f[1].D) * (f[0].r2 * f[1].r2);  // dd2(0, 1)
    const T v2 = T(4) * (f[0].D * f[2].D) * (f[0].r2 * f[2].r2);  // dd2(0, 2)
    const T v3 = T(4) * (f[0].D * f[3].D) * (f[0].r2 * f[3].r2);  // dd2(0, 3)
    const T v4 = f[1].DD1;  // dd1(1,)
    const T v5 = T(4) * (f[1].D * f[2].D) * (f[1].r2 * f[2].r2);  // dd2(1, 2)
    const T v6 = T(4) * (f[1].D * f[3].D) * (f[1].r2 * f[3].r2);  // dd2(1, 3)
    const T v7 = f[2].DD1;  // dd1(2,)
    const T v8 = T(4) * (f[2].D * f[3].D) * (f[2].r2 * f[3].r2);  // dd2(2, 3)
    const T v9 = f[3].DD1;  // dd1(3,)
    const T v10 = f[0].DZ1;  // dz_iii(0,)
    const T v11 = (T(2) * f[0].U * f[1].A) * (f[0].u3 * f[1].u1);  // dz_iij(0, 1)
    const T v12 = (T(2) * f[0].V * f[1].Bv) * (f[0].u3 * f[1].u1);  // dz_iji(0, 1)
    const T v13 = (T(2) * f[0].U * f[2].A) * (f[0].u3 * f[2].u1);  // dz_iij(0, 2)
    const T v14 = (T(2) * f[0].V * f[2].Bv) * (f[0].u3 * f[2].u1);  // dz_iji(0, 2)
    const T v15 = (T(2) * f[0].U * f[3].A) * (f[0].u3 * f[3].u1);  // dz_iij(0, 3)
    const T v16 = (T(2) * f[0].V * f[3].Bv) * (f[0].u3 * f[3].u1);  // dz_iji(0, 3)
    const T v17 = (T(2) * f[0].D * f[1].Wjj) * (f[1].u2 * f[0].u2);  // dz_ijj(0, 1)
    const T v18 = (T(2) * f[0].D * f[1].Bv * f[2].A) * (f[0].u2 * f[1].u1 * f[2].u1);  // dz_ijk(0, 1, 2)
    const T v19 = (T(2) * f[0].D * f[2].Bv * f[1].A) * (f[0].u2 * f[2].u1 * f[1].u1);  // dz_ijk(0, 2, 1)
    const T v20 = (T(2) * f[0].D * f[1].Bv * f[3].A) * (f[0].u2 * f[1].u1 * f[3].u1);  // dz_ijk(0, 1, 3)
    const T v21 = (T(2) * f[0].D * f[3].Bv * f[1].A) * (f[0].u2 * f[3].u1 * f[1].u1);  // dz_ijk(0, 3, 1)
    const T v22 = (T(2) * f[0].D * f[2].Wjj) * (f[2].u2 * f[0].u2);  // dz_ijj(0, 2)
    const T v23 = (T(2) * f[0].D * f[2].Bv * f[3].A) * (f[0].u2 * f[2].u1 * f[3].u1);  // dz_ijk(0, 2, 3)
    const T v24 = (T(2) * f[0].D * f[3].Bv * f[2].A) * (f[0].u2 * f[3].u1 * f[2].u1);  // dz_ijk(0, 3, 2)
    const T v25 = (T(2) * f[0].D * f[3].Wjj) * (f[3].u2 * f[0].u2);  // dz_ijj(0, 3)
    const T v26 = (T(2) * f[1].D * f[0].Wjj) * (f[0].u2 * f[1].u2);  // dz_ijj(1, 0)
    const T v27 = (T(2) * f[1].V * f[0].Bv) * (f[1].u3 * f[0].u1);  // dz_iji(1, 0)
    const T v28 = (T(2) * f[1].U * f[0].A) * (f[1].u3 * f[0].u1);  // dz_iij(1, 0)
    const T v29 = (T(2) * f[1].D * f[0].Bv * f[2].A) * (f[1].u2 * f[0].u1 * f[2].u1);  // dz_ijk(1, 0, 2)
    const T v30 = (T(2) * f[1].D * f[2].Bv * f[0].A) * (f[1].u2 * f[2].u1 * f[0].u1);  // dz_ijk(1, 2, 0)
    const T v31 = (T(2) * f[1].D * f[0].Bv * f[3].A) * (f[1].u2 * f[0].u1 * f[3].u1);  // dz_ijk(1, 0, 3)
    const T v32 = (T(2) * f[1].D * f[3].Bv * f[0].A) * (f[1].u2 * f[3].u1 * f[0].u1);  // dz_ijk(1, 3, 0)
    const T v33 = f[1].DZ1;  // dz_iii(1,)
    const T v34 = (T(2) * f[1].U * f[2].A) * (f[1].u3 * f[2].u1);  // dz_iij(1, 2)
    const T v35 = (T(2) * f[1].V * f[2].Bv) * (f[1].u3 * f[2].u1);  // dz_iji(1, 2)
    const T v36 = (T(2) * f[1].U * f[3].A) * (f[1].u3 * f[3].u1);  // dz_iij(1, 3)
    const T v37 = (T(2) * f[1].V * f[3].Bv) * (f[1].u3 * f[3].u1);  // dz_iji(1, 3)
    const T v38 = (T(2) * f[1].D * f[2].Wjj) * (f[2].u2 * f[1].u2);  // dz_ijj(1, 2)
    const T v39 = (T(2) * f[1].D * f[2].Bv * f[3].A) * (f[1].u2 * f[2].u1 * f[3].u1);  // dz_ijk(1, 2, 3)
    const T v40 = (T(2) * f[1].D * f[3].Bv * f[2].A) * (f[1].u2 * f[3].u1 * f[2].u1);  // dz_ijk(1, 3, 2)
    const T v41 = (T(2) * f[1].D * f[3].Wjj) * (f[3].u2 * f[1].u2);  // dz_ijj(1, 3)
    const T v42 = (T(2) * f[2].D * f[0].Wjj) * (f[0].u2 * f[2].u2);  // dz_ijj(2, 0)
    const T v43 = (T(2) * f[2].D * f[0].Bv * f[1].A) * (f[2].u2 * f[0].u1 * f[1].u1);  // dz_ijk(2, 0, 1)
    const T v44 = (T(2) * f[2].D * f[1].Bv * f[0].A) * (f[2].u2 * f[1].u1 * f[0].u1);  // dz_ijk(2, 1, 0)
    const T v45 = (T(2) * f[2].V * f[0].Bv) * (f[2].u3 * f[0].u1);  // dz_iji(2, 0)
    const T v46 = (T(2) * f[2].U * f[0].A) * (f[2].u3 * f[0].u1);  // dz_iij(2, 0)
    const T v47 = (T(2) * f[2].D * f[0].Bv * f[3].A) * (f[2].u2 * f[0].u1 * f[3].u1);  // dz_ijk(2, 0, 3)
    const T v48 = (T(2) * f[2].D * f[3].Bv * f[0].A) * (f[2].u2 * f[3].u1 * f[0].u1);  // dz_ijk(2, 3, 0)
    const T v49 = (T(2) * f[2].D * f[1].Wjj) * (f[1].u2 * f[2].u2);  // dz_ijj(2, 1)
    const T v50 = (T(2) * f[2].V * f[1].Bv) * (f[2].u3 * f[1].u1);  // dz_iji(2, 1)
    const T v51 = (T(2) * f[2].U * f[1].A) * (f[2].u3 * f[1].u1);  // dz_iij(2, 1)
    const T v52 = (T(2) * f[2].D * f[1].Bv * f[3].A) * (f[2].u2 * f[1].u1 * f[3].u1);  // dz_ijk(2, 1, 3)
    const T v53 = (T(2) * f[2].D * f[3].Bv * f[1].A) * (f[2].u2 * f[3].u1 * f[1].u1);  // dz_ijk(2, 3, 1)
    const T v54 = f[2].DZ1;  // dz_iii(2,)
    const T v55 = (T(2) * f[2].U * f[3].A) * (f[2].u3 * f[3].u1);  // dz_iij(2, 3)
    const T v56 = (T(2) * f[2].V * f[3].Bv) * (f[2].u3 * f[3].u1);  // dz_iji(2, 3)
    const T v57 = (T(2) * f[2].D * f[3].Wjj) * (f[3].u2 * f[2].u2);  // dz_ijj(2, 3)
    const T v58 = (T(2) * f[3].D * f[0].Wjj) * (f[0].u2 * f[3].u2);  // dz_ijj(3, 0)
    const T v59 = (T(2) * f[3].D * f[0].Bv * f[1].A) * (f[3].u2 * f[0].u1 * f[1].u1);  // dz_ijk(3, 0, 1)
    const T v60 = (T(2) * f[3].D * f[1].Bv * f[0].A) * (f[3].u2 * f[1].u1 * f[0].u1);  // dz_ijk(3, 1, 0)
    const T v61 = (T(2) * f[3].D * f[0].Bv * f[2].A) * (f[3].u2 * f[0].u1 * f[2].u1);  // dz_ijk(3, 0, 2)
    const T v62 = (T(2) * f[3].D * f[2].Bv * f[0].A) * (f[3].u2 * f[2].u1 * f[0].u1);  // dz_ijk(3, 2, 0)
    const T v63 = (T(2) * f[3].V * f[0].Bv) * (f[3].u3 * f[0].u1);  // dz_iji(3, 0)
    const T v64 = (T(2) * f[3].U * f[0].A) * (f[3].u3 * f[0].u1);  // dz_iij(3, 0)
    const T v65 = (T(2) * f[3].D * f[1].Wjj) * (f[1].u2 * f[3].u2);  // dz_ijj(3, 1)
    const T v66 = (T(2) * f[3].D * f[1].Bv * f[2].A) * (f[3].u2 * f[1].u1 * f[2].u1);  // dz_ijk(3, 1, 2)
    const T v67 = (T(2) * f[3].D * f[2].Bv * f[1].A) * (f[3].u2 * f[2].u1 * f[1].u1);  // dz_ijk(3, 2, 1)
    const T v68 = (T(2) * f[3].V * f[1].Bv) * (f[3].u3 * f[1].u1);  // dz_iji(3, 1)
    const T v69 = (T(2) * f[3].U * f[1].A) * (f[3].u3 * f[1].u1);  // dz_iij(3, 1)
    const T v70 = (T(2) * f[3].D * f[2].Wjj) * (f[2].u2 * f[3].u2);  // dz_ijj(3, 2)
    const T v71 = (T(2) * f[3].V * f[2].Bv) * (f[3].u3 * f[2].u1);  // dz_iji(3, 2)
    const T v72 = (T(2) * f[3].U * f[2].A) * (f[3].u3 * f[2].u1);  // dz_iij(3, 2)
    const T v73 = f[3].DZ1;  // dz_iii(3,)
    const T v74 = f[0].PI1;  // pi2_same(0,)
    const T v75 = (f[0].AQ3 * f[1].pB + f[0].AS3 * f[1].qB) * (f[0].r3 * f[1].r1);  // pi2_iiij(0, 1)
    const T v76 = (f[0].BP3 * f[1].pA + f[0].BR3 * f[1].qA) * (f[0].r3 * f[1].r1);  // pi2_ijii(0, 1)
    const T v77 = (f[0].AQ3 * f[2].pB + f[0].AS3 * f[2].qB) * (f[0].r3 * f[2].r1);  // pi2_iiij(0, 2)
    const T v78 = (f[0].BP3 * f[2].pA + f[0].BR3 * f[2].qA) * (f[0].r3 * f[2].r1);  // pi2_ijii(0, 2)
    const T v79 = (f[0].AQ3 * f[3].pB + f[0].AS3 * f[3].qB) * (f[0].r3 * f[3].r1);  // pi2_iiij(0, 3)
    const T v80 = (f[0].BP3 * f[3].pA + f[0].BR3 * f[3].qA) * (f[0].r3 * f[3].r1);  // pi2_ijii(0, 3)
    const T v81 = f[0].BL * f[1].BR;  // pi2_iikk(0, 1)
    const T v82 = f[1].BL * f[0].BR;  // pi2_iikk(1, 0)
    const T v83 = f[0].BL * T(0.5) * (f[1].q * f[2].s + f[1].s * f[2].q);  // pi2_iikl(0, 1, 2)
    const T v84 = T(0.5) * (f[1].p * f[2].r + f[1].r * f[2].p) * f[0].BR;  // pi2_ijkk(1, 2, 0)
    const T v85 = f[0].BL * T(0.5) * (f[1].q * f[3].s + f[1].s * f[3].q);  // pi2_iikl(0, 1, 3)
    const T v86 = T(0.5) * (f[1].p * f[3].r + f[1].r * f[3].p) * f[0].BR;  // pi2_ijkk(1, 3, 0)
    const T v87 = f[0].BL * f[2].BR;  // pi2_iikk(0, 2)
    const T v88 = f[2].BL * f[0].BR;  // pi2_iikk(2, 0)
    const T v89 = f[0].BL * T(0.5) * (f[2].q * f[3].s + f[2].s * f[3].q);  // pi2_iikl(0, 2, 3)
    const T v90 = T(0.5) * (f[2].p * f[3].r + f[2].r * f[3].p) * f[0].BR;  // pi2_ijkk(2, 3, 0)
    const T v91 = f[0].BL * f[3].BR;  // pi2_iikk(0, 3)
    const T v92 = f[3].BL * f[0].BR;  // pi2_iikk(3, 0)
    const T v93 = (-T(0.25) * (f[0].qA * f[0].qB) * f[1].pB - T(0.25) * f[0].xab * (f[1].pA * f[1].pB) + T(0.25) * (f[0].qA * f[0].qB) * (f[1].pA * f[1].pB) - T(0.25) * f[0].qA * (f[1].pA * f[1].qB) - T(0.25) * (f[0].pA * f[0].pB) * f[1].xab - T(0.25) * (f[0].qA * f[0].qB) * f[1].xab + T(0.25) * (f[0].pA * f[0].qB) * f[1].xab + T(0.25) * (f[0].pB * f[0].qA) * f[1].xab - T(0.25) * (f[0].pA * f[0].qA) * f[1].qB + T(0.25) * (f[0].qA * (T(1) + f[0].xAb - f[0].xaB)) * f[1].qB + T(0.25) * f[0].xab * (f[1].pA * f[1].qB) + T(0.25) * (f[0].pB * f[0].qA) * (f[1].pA * f[1].qB) + T(0.25) * (f[0].qB * (T(1) + f[0].qA)) * f[1].qA - T(0.25) * f[0].xAb * (f[1].pB * f[1].qA) + T(0.25) * (f[0].pA * f[0].qB) * (f[1].pB * f[1].qA) - T(0.25) * (f[0].pA * f[0].qB) * f[1].qA - T(0.25) * f[0].pA * (f[1].qA * f[1].qB) + T(0.25) * f[0].xAb * (f[1].qA * f[1].qB) + T(0.25) * (f[0].pA * f[0].pB) * (f[1].qA * f[1].qB) + T(0.25) * f[0].xab * f[1].Bsgn + T(0.25) * f[0].Bsgn * f[1].xab - f[0].xab * f[1].xab) * (f[0].r2 * f[1].r2);  // pi2_ijij(0, 1)
    const T v94 = (-T(0.25) * (f[1].qA * f[1].qB) * f[0].pB - T(0.25) * f[1].xab * (f[0].pA * f[0].pB) + T(0.25) * (f[1].qA * f[1].qB) * (f[0].pA * f[0].pB) - T(0.25) * f[1].qA * (f[0].pA * f[0].qB) - T(0.25) * (f[1].pA * f[1].pB) * f[0].xab - T(0.25) * (f[1].qA * f[1].qB) * f[0].xab + T(0.25) * (f[1].pA * f[1].qB) * f[0].xab + T(0.25) * (f[1].pB * f[1].qA) * f[0].xab - T(0.25) * (f[1].pA * f[1].qA) * f[0].qB + T(0.25) * (f[1].qA * (T(1) + f[1].xAb - f[1].xaB)) * f[0].qB + T(0.25) * f[1].xab * (f[0].pA * f[0].qB) + T(0.25) * (f[1].pB * f[1].qA) * (f[0].pA * f[0].qB) + T(0.25) * (f[1].qB * (T(1) + f[1].qA)) * f[0].qA - T(0.25) * f[1].xAb * (f[0].pB * f[0].qA) + T(0.25) * (f[1].pA * f[1].qB) * (f[0].pB * f[0].qA) - T(0.25) * (f[1].pA * f[1].qB) * f[0].qA - T(0.25) * f[1].pA * (f[0].qA * f[0].qB) + T(0.25) * f[1].xAb * (f[0].qA * f[0].qB) + T(0.25) * (f[1].pA * f[1].pB) * (f[0].qA * f[0].qB) + T(0.25) * f[1].xab * f[0].Bsgn + T(0.25) * f[1].Bsgn * f[0].xab - f[1].xab * f[0].xab) * (f[1].r2 * f[0].r2);  // pi2_ijij(1, 0)
    const T v95 = f[1].r * (f[0].C00 * f[2].s + f[0].C01 * f[2].q) + f[1].p * (f[0].C10 * f[2].s + f[0].C11 * f[2].q);  // pi2_shared(0, 1, 2)
    const T v96 = f[2].r * (f[0].C00 * f[1].s + f[0].C01 * f[1].q) + f[2].p * (f[0].C10 * f[1].s + f[0].C11 * f[1].q);  // pi2_shared(0, 2, 1)
    const T v97 = f[1].r * (f[0].C00 * f[3].s + f[0].C01 * f[3].q) + f[1].p * (f[0].C10 * f[3].s + f[0].C11 * f[3].q);  // pi2_shared(0, 1, 3)
    const T v98 = f[3].r * (f[0].C00 * f[1].s + f[0].C01 * f[1].q) + f[3].p * (f[0].C10 * f[1].s + f[0].C11 * f[1].q);  // pi2_shared(0, 3, 1)
    const T v99 = (f[1].BP3 * f[0].pA + f[1].BR3 * f[0].qA) * (f[1].r3 * f[0].r1);  // pi2_ijii(1, 0)
    const T v100 = (f[1].AQ3 * f[0].pB + f[1].AS3 * f[0].qB) * (f[1].r3 * f[0].r1);  // pi2_iiij(1, 0)
    const T v101 = f[0].r * (f[1].C00 * f[2].s + f[1].C01 * f[2].q) + f[0].p * (f[1].C10 * f[2].s + f[1].C11 * f[2].q);  // pi2_shared(1, 0, 2)
    const T v102 = f[2].r * (f[1].C00 * f[0].s + f[1].C01 * f[0].q) + f[2].p * (f[1].C10 * f[0].s + f[1].C11 * f[0].q);  // pi2_shared(1, 2, 0)
    const T v103 = f[0].r * (f[1].C00 * f[3].s + f[1].C01 * f[3].q) + f[0].p * (f[1].C10 * f[3].s + f[1].C11 * f[3].q);  // pi2_shared(1, 0, 3)
    const T v104 = f[3].r * (f[1].C00 * f[0].s + f[1].C01 * f[0].q) + f[3].p * (f[1].C10 * f[0].s + f[1].C11 * f[0].q);  // pi2_shared(1, 3, 0)
    const T v105 = T(0.5) * (f[0].p * f[1].r + f[0].r * f[1].p) * f[2].BR;  // pi2_ijkk(0, 1, 2)
    const T v106 = f[2].BL * T(0.5) * (f[0].q * f[1].s + f[0].s * f[1].q);  // pi2_iikl(2, 0, 1)
    const T v107 = T(0.25) * (f[0].p * f[1].r + f[0].r * f[1].p) * (f[2].q * f[3].s + f[2].s * f[3].q);  // pi2_alldiff(0, 1, 2, 3)
    const T v108 = T(0.25) * (f[2].p * f[3].r + f[2].r * f[3].p) * (f[0].q * f[1].s + f[0].s * f[1].q);  // pi2_alldiff(2, 3, 0, 1)
    const T v109 = T(0.5) * (f[0].p * f[1].r + f[0].r * f[1].p) * f[3].BR;  // pi2_ijkk(0, 1, 3)
    const T v110 = f[3].BL * T(0.5) * (f[0].q * f[1].s + f[0].s * f[1].q);  // pi2_iikl(3, 0, 1)
    const T v111 = (-T(0.25) * (f[0].qA * f[0].qB) * f[2].pB - T(0.25) * f[0].xab * (f[2].pA * f[2].pB) + T(0.25) * (f[0].qA * f[0].qB) * (f[2].pA * f[2].pB) - T(0.25) * f[0].qA * (f[2].pA * f[2].qB) - T(0.25) * (f[0].pA * f[0].pB) * f[2].xab - T(0.25) * (f[0].qA * f[0].qB) * f[2].xab + T(0.25) * (f[0].pA * f[0].qB) * f[2].xab + T(0.25) * (f[0].pB * f[0].qA) * f[2].xab - T(0.25) * (f[0].pA * f[0].qA) * f[2].qB + T(0.25) * (f[0].qA * (T(1) + f[0].xAb - f[0].xaB)) * f[2].qB + T(0.25) * f[0].xab * (f[2].pA * f[2].qB) + T(0.25) * (f[0].pB * f[0].qA) * (f[2].pA * f[2].qB) + T(0.25) * (f[0].qB * (T(1) + f[0].qA)) * f[2].qA - T(0.25) * f[0].xAb * (f[2].pB * f[2].qA) + T(0.25) * (f[0].pA * f[0].qB) * (f[2].pB * f[2].qA) - T(0.25) * (f[0].pA * f[0].qB) * f[2].qA - T(0.25) * f[0].pA * (f[2].qA * f[2].qB) + T(0.25) * f[0].xAb * (f[2].qA * f[2].qB) + T(0.25) * (f[0].pA * f[0].pB) * (f[2].qA * f[2].qB) + T(0.25) * f[0].xab * f[2].Bsgn + T(0.25) * f[0].Bsgn * f[2].xab - f[0].xab * f[2].xab) * (f[0].r2 * f[2].r2);  // pi2_ijij(0, 2)
    const T v112 = (-T(0.25) * (f[2].qA * f[2].qB) * f[0].pB - T(0.25) * f[2].xab * (f[0].pA * f[0].pB) + T(0.25) * (f[2].qA * f[2].qB) * (f[0].pA * f[0].pB) - T(0.25) * f[2].qA * (f[0].pA * f[0].qB) - T(0.25) * (f[2].pA * f[2].pB) * f[0].xab - T(0.25) * (f[2].qA * f[2].qB) * f[0].xab + T(0.25) * (f[2].pA * f[2].qB) * f[0].xab + T(0.25) * (f[2].pB * f[2].qA) * f[0].xab - T(0.25) * (f[2].pA * f[2].qA) * f[0].qB + T(0.25) * (f[2].qA * (T(1) + f[2].xAb - f[2].xaB)) * f[0].qB + T(0.25) * f[2].xab * (f[0].pA * f[0].qB) + T(0.25) * (f[2].pB * f[2].qA) * (f[0].pA * f[0].qB) + T(0.25) * (f[2].qB * (T(1) + f[2].qA)) * f[0].qA - T(0.25) * f[2].xAb * (f[0].pB * f[0].qA) + T(0.25) * (f[2].pA * f[2].qB) * (f[0].pB * f[0].qA) - T(0.25) * (f[2].pA * f[2].qB) * f[0].qA - T(0.25) * f[2].pA * (f[0].qA * f[0].qB) + T(0.25) * f[2].xAb * (f[0].qA * f[0].qB) + T(0.25) * (f[2].pA * f[2].pB) * (f[0].qA * f[0].qB) + T(0.25) * f[2].xab * f[0].Bsgn + T(0.25) * f[2].Bsgn * f[0].xab - f[2].xab * f[0].xab) * (f[2].r2 * f[0].r2);  // pi2_ijij(2, 0)
    const T v113 = f[2].r * (f[0].C00 * f[3].s + f[0].C01 * f[3].q) + f[2].p * (f[0].C10 * f[3].s + f[0].C11 * f[3].q);  // pi2_shared(0, 2, 3)
    const T v114 = f[3].r * (f[0].C00 * f[2].s + f[0].C01 * f[2].q) + f[3].p * (f[0].C10 * f[2].s + f[0].C11 * f[2].q);  // pi2_shared(0, 3, 2)
    const T v115 = T(0.5) * (f[0].p * f[2].r + f[0].r * f[2].p) * f[1].BR;  // pi2_ijkk(0, 2, 1)
    const T v116 = f[1].BL * T(0.5) * (f[0].q * f[2].s + f[0].s * f[2].q);  // pi2_iikl(1, 0, 2)
    const T v117 = f[0].r * (f[2].C00 * f[1].s + f[2].C01 * f[1].q) + f[0].p * (f[2].C10 * f[1].s + f[2].C11 * f[1].q);  // pi2_shared(2, 0, 1)
    const T v118 = f[1].r * (f[2].C00 * f[0].s + f[2].C01 * f[0].q) + f[1].p * (f[2].C10 * f[0].s + f[2].C11 * f[0].q);  // pi2_shared(2, 1, 0)
    const T v119 = T(0.25) * (f[0].p * f[2].r + f[0].r * f[2].p) * (f[1].q * f[3].s + f[1].s * f[3].q);  // pi2_alldiff(0, 2, 1, 3)
    const T v120 = T(0.25) * (f[1].p * f[3].r + f[1].r * f[3].p) * (f[0].q * f[2].s + f[0].s * f[2].q);  // pi2_alldiff(1, 3, 0, 2)
    const T v121 = (f[2].BP3 * f[0].pA + f[2].BR3 * f[0].qA) * (f[2].r3 * f[0].r1);  // pi2_ijii(2, 0)
    const T v122 = (f[2].AQ3 * f[0].pB + f[2].AS3 * f[0].qB) * (f[2].r3 * f[0].r1);  // pi2_iiij(2, 0)
    const T v123 = f[0].r * (f[2].C00 * f[3].s + f[2].C01 * f[3].q) + f[0].p * (f[2].C10 * f[3].s + f[2].C11 * f[3].q);  // pi2_shared(2, 0, 3)
    const T v124 = f[3].r * (f[2].C00 * f[0].s + f[2].C01 * f[0].q) + f[3].p * (f[2].C10 * f[0].s + f[2].C11 * f[0].q);  // pi2_shared(2, 3, 0)
    const T v125 = T(0.5) * (f[0].p * f[2].r + f[0].r * f[2].p) * f[3].BR;  // pi2_ijkk(0, 2, 3)
    const T v126 = f[3].BL * T(0.5) * (f[0].q * f[2].s + f[0].s * f[2].q);  // pi2_iikl(3, 0, 2)
    const T v127 = (-T(0.25) * (f[0].qA * f[0].qB) * f[3].pB - T(0.25) * f[0].xab * (f[3].pA * f[3].pB) + T(0.25) * (f[0].qA * f[0].qB) * (f[3].pA * f[3].pB) - T(0.25) * f[0].qA * (f[3].pA * f[3].qB) - T(0.25) * (f[0].pA * f[0].pB) * f[3].xab - T(0.25) * (f[0].qA * f[0].qB) * f[3].xab + T(0.25) * (f[0].pA * f[0].qB) * f[3].xab + T(0.25) * (f[0].pB * f[0].qA) * f[3].xab - T(0.25) * (f[0].pA * f[0].qA) * f[3].qB + T(0.25) * (f[0].qA * (T(1) + f[0].xAb - f[0].xaB)) * f[3].qB + T(0.25) * f[0].xab * (f[3].pA * f[3].qB) + T(0.25) * (f[0].pB * f[0].qA) * (f[3].pA * f[3].qB) + T(0.25) * (f[0].qB * (T(1) + f[0].qA)) * f[3].qA - T(0.25) * f[0].xAb * (f[3].pB * f[3].qA) + T(0.25) * (f[0].pA * f[0].qB) * (f[3].pB * f[3].qA) - T(0.25) * (f[0].pA * f[0].qB) * f[3].qA - T(0.25) * f[0].pA * (f[3].qA * f[3].qB) + T(0.25) * f[0].xAb * (f[3].qA * f[3].qB) + T(0.25) * (f[0].pA * f[0].pB) * (f[3].qA * f[3].qB) + T(0.25) * f[0].xab * f[3].Bsgn + T(0.25) * f[0].Bsgn * f[3].xab - f[0].xab * f[3].xab) * (f[0].r2 * f[3].r2);  // pi2_ijij(0, 3)
    const T v128 = (-T(0.25) * (f[3].qA * f[3].qB) * f[0].pB - T(0.25) * f[3].xab * (f[0].pA * f[0].pB) + T(0.25) * (f[3].qA * f[3].qB) * (f[0].pA * f[0].pB) - T(0.25) * f[3].qA * (f[0].pA * f[0].qB) - T(0.25) * (f[3].pA * f[3].pB) * f[0].xab - T(0.25) * (f[3].qA * f[3].qB) * f[0].xab + T(0.25) * (f[3].pA * f[3].qB) * f[0].xab + T(0.25) * (f[3].pB * f[3].qA) * f[0].xab - T(0.25) * (f[3].pA * f[3].qA) * f[0].qB + T(0.25) * (f[3].qA * (T(1) + f[3].xAb - f[3].xaB)) * f[0].qB + T(0.25) * f[3].xab * (f[0].pA * f[0].qB) + T(0.25) * (f[3].pB * f[3].qA) * (f[0].pA * f[0].qB) + T(0.25) * (f[3].qB * (T(1) + f[3].qA)) * f[0].qA - T(0.25) * f[3].xAb * (f[0].pB * f[0].qA) + T(0.25) * (f[3].pA * f[3].qB) * (f[0].pB * f[0].qA) - T(0.25) * (f[3].pA * f[3].qB) * f[0].qA - T(0.25) * f[3].pA * (f[0].qA * f[0].qB) + T(0.25) * f[3].xAb * (f[0].qA * f[0].qB) + T(0.25) * (f[3].pA * f[3].pB) * (f[0].qA * f[0].qB) + T(0.25) * f[3].xab * f[0].Bsgn + T(0.25) * f[3].Bsgn * f[0].xab - f[3].xab * f[0].xab) * (f[3].r2 * f[0].r2);  // pi2_ijij(3, 0)
    const T v129 = T(0.5) * (f[0].p * f[3].r + f[0].r * f[3].p) * f[1].BR;  // pi2_ijkk(0, 3, 1)
    const T v130 = f[1].BL * T(0.5) * (f[0].q * f[3].s + f[0].s * f[3].q);  // pi2_iikl(1, 0, 3)
    const T v131 = T(0.25) * (f[0].p * f[3].r + f[0].r * f[3].p) * (f[1].q * f[2].s + f[1].s * f[2].q);  // pi2_alldiff(0, 3, 1, 2)
    const T v132 = T(0.25) * (f[1].p * f[2].r + f[1].r * f[2].p) * (f[0].q * f[3].s + f[0].s * f[3].q);  // pi2_alldiff(1, 2, 0, 3)
    const T v133 = f[0].r * (f[3].C00 * f[1].s + f[3].C01 * f[1].q) + f[0].p * (f[3].C10 * f[1].s + f[3].C11 * f[1].q);  // pi2_shared(3, 0, 1)
    const T v134 = f[1].r * (f[3].C00 * f[0].s + f[3].C01 * f[0].q) + f[1].p * (f[3].C10 * f[0].s + f[3].C11 * f[0].q);  // pi2_shared(3, 1, 0)
    const T v135 = T(0.5) * (f[0].p * f[3].r + f[0].r * f[3].p) * f[2].BR;  // pi2_ijkk(0, 3, 2)
    const T v136 = f[2].BL * T(0.5) * (f[0].q * f[3].s + f[0].s * f[3].q);  // pi2_iikl(2, 0, 3)
    const T v137 = f[0].r * (f[3].C00 * f[2].s + f[3].C01 * f[2].q) + f[0].p * (f[3].C10 * f[2].s + f[3].C11 * f[2].q);  // pi2_shared(3, 0, 2)
    const T v138 = f[2].r * (f[3].C00 * f[0].s + f[3].C01 * f[0].q) + f[2].p * (f[3].C10 * f[0].s + f[3].C11 * f[0].q);  // pi2_shared(3, 2, 0)
    const T v139 = (f[3].BP3 * f[0].pA + f[3].BR3 * f[0].qA) * (f[3].r3 * f[0].r1);  // pi2_ijii(3, 0)
    const T v140 = (f[3].AQ3 * f[0].pB + f[3].AS3 * f[0].qB) * (f[3].r3 * f[0].r1);  // pi2_iiij(3, 0)
    const T v141 = f[1].PI1;  // pi2_same(1,)
    const T v142 = (f[1].AQ3 * f[2].pB + f[1].AS3 * f[2].qB) * (f[1].r3 * f[2].r1);  // pi2_iiij(1, 2)
    const T v143 = (f[1].BP3 * f[2].pA + f[1].BR3 * f[2].qA) * (f[1].r3 * f[2].r1);  // pi2_ijii(1, 2)
    const T v144 = (f[1].AQ3 * f[3].pB + f[1].AS3 * f[3].qB) * (f[1].r3 * f[3].r1);  // pi2_iiij(1, 3)
    const T v145 = (f[1].BP3 * f[3].pA + f[1].BR3 * f[3].qA) * (f[1].r3 * f[3].r1);  // pi2_ijii(1, 3)
    const T v146 = f[1].BL * f[2].BR;  // pi2_iikk(1, 2)
    const T v147 = f[2].BL * f[1].BR;  // pi2_iikk(2, 1)
    const T v148 = f[1].BL * T(0.5) * (f[2].q * f[3].s + f[2].s * f[3].q);  // pi2_iikl(1, 2, 3)
    const T v149 = T(0.5) * (f[2].p * f[3].r + f[2].r * f[3].p) * f[1].BR;  // pi2_ijkk(2, 3, 1)
    const T v150 = f[1].BL * f[3].BR;  // pi2_iikk(1, 3)
    const T v151 = f[3].BL * f[1].BR;  // pi2_iikk(3, 1)
    const T v152 = (-T(0.25) * (f[1].qA * f[1].qB) * f[2].pB - T(0.25) * f[1].xab * (f[2].pA * f[2].pB) + T(0.25) * (f[1].qA * f[1].qB) * (f[2].pA * f[2].pB) - T(0.25) * f[1].qA * (f[2].pA * f[2].qB) - T(0.25) * (f[1].pA * f[1].pB) * f[2].xab - T(0.25) * (f[1].qA * f[1].qB) * f[2].xab + T(0.25) * (f[1].pA * f[1].qB) * f[2].xab + T(0.25) * (f[1].pB * f[1].qA) * f[2].xab - T(0.25) * (f[1].pA * f[1].qA) * f[2].qB + T(0.25) * (f[1].qA * (T(1) + f[1].xAb - f[1].xaB)) * f[2].qB + T(0.25) * f[1].xab * (f[2].pA * f[2].qB) + T(0.25) * (f[1].pB * f[1].qA) * (f[2].pA * f[2].qB) + T(0.25) * (f[1].qB * (T(1) + f[1].qA)) * f[2].qA - T(0.25) * f[1].xAb * (f[2].pB * f[2].qA) + T(0.25) * (f[1].pA * f[1].qB) * (f[2].pB * f[2].qA) - T(0.25) * (f[1].pA * f[1].qB) * f[2].qA - T(0.25) * f[1].pA * (f[2].qA * f[2].qB) + T(0.25) * f[1].xAb * (f[2].qA * f[2].qB) + T(0.25) * (f[1].pA * f[1].pB) * (f[2].qA * f[2].qB) + T(0.25) * f[1].xab * f[2].Bsgn + T(0.25) * f[1].Bsgn * f[2].xab - f[1].xab * f[2].xab) * (f[1].r2 * f[2].r2);  // pi2_ijij(1, 2)
    const T v153 = (-T(0.25) * (f[2].qA * f[2].qB) * f[1].pB - T(0.25) * f[2].xab * (f[1].pA * f[1].pB) + T(0.25) * (f[2].qA * f[2].qB) * (f[1].pA * f[1].pB) - T(0.25) * f[2].qA * (f[1].pA * f[1].qB) - T(0.25) * (f[2].pA * f[2].pB) * f[1].xab - T(0.25) * (f[2].qA * f[2].qB) * f[1].xab + T(0.25) * (f[2].pA * f[2].qB) * f[1].xab + T(0.25) * (f[2].pB * f[2].qA) * f[1].xab - T(0.25) * (f[2].pA * f[2].qA) * f[1].qB + T(0.25) * (f[2].qA * (T(1) + f[2].xAb - f[2].xaB)) * f[1].qB + T(0.25) * f[2].xab * (f[1].pA * f[1].qB) + T(0.25) * (f[2].pB * f[2].qA) * (f[1].pA * f[1].qB) + T(0.25) * (f[2].qB * (T(1) + f[2].qA)) * f[1].qA - T(0.25) * f[2].xAb * (f[1].pB * f[1].qA) + T(0.25) * (f[2].pA * f[2].qB) * (f[1].pB * f[1].qA) - T(0.25) * (f[2].pA * f[2].qB) * f[1].qA - T(0.25) * f[2].pA * (f[1].qA * f[1].qB) + T(0.25) * f[2].xAb * (f[1].qA * f[1].qB) + T(0.25) * (f[2].pA * f[2].pB) * (f[1].qA * f[1].qB) + T(0.25) * f[2].xab * f[1].Bsgn + T(0.25) * f[2].Bsgn * f[1].xab - f[2].xab * f[1].xab) * (f[2].r2 * f[1].r2);  // pi2_ijij(2, 1)
    const T v154 = f[2].r * (f[1].C00 * f[3].s + f[1].C01 * f[3].q) + f[2].p * (f[1].C10 * f[3].s + f[1].C11 * f[3].q);  // pi2_shared(1, 2, 3)
    const T v155 = f[3].r * (f[1].C00 * f[2].s + f[1].C01 * f[2].q) + f[3].p * (f[1].C10 * f[2].s + f[1].C11 * f[2].q);  // pi2_shared(1, 3, 2)
    const T v156 = (f[2].BP3 * f[1].pA + f[2].BR3 * f[1].qA) * (f[2].r3 * f[1].r1);  // pi2_ijii(2, 1)
    const T v157 = (f[2].AQ3 * f[1].pB + f[2].AS3 * f[1].qB) * (f[2].r3 * f[1].r1);  // pi2_iiij(2, 1)
    const T v158 = f[1].r * (f[2].C00 * f[3].s + f[2].C01 * f[3].q) + f[1].p * (f[2].C10 * f[3].s + f[2].C11 * f[3].q);  // pi2_shared(2, 1, 3)
    const T v159 = f[3].r * (f[2].C00 * f[1].s + f[2].C01 * f[1].q) + f[3].p * (f[2].C10 * f[1].s + f[2].C11 * f[1].q);  // pi2_shared(2, 3, 1)
    const T v160 = T(0.5) * (f[1].p * f[2].r + f[1].r * f[2].p) * f[3].BR;  // pi2_ijkk(1, 2, 3)
    const T v161 = f[3].BL * T(0.5) * (f[1].q * f[2].s + f[1].s * f[2].q);  // pi2_iikl(3, 1, 2)
    const T v162 = (-T(0.25) * (f[1].qA * f[1].qB) * f[3].pB - T(0.25) * f[1].xab * (f[3].pA * f[3].pB) + T(0.25) * (f[1].qA * f[1].qB) * (f[3].pA * f[3].pB) - T(0.25) * f[1].qA * (f[3].pA * f[3].qB) - T(0.25) * (f[1].pA * f[1].pB) * f[3].xab - T(0.25) * (f[1].qA * f[1].qB) * f[3].xab + T(0.25) * (f[1].pA * f[1].qB) * f[3].xab + T(0.25) * (f[1].pB * f[1].qA) * f[3].xab - T(0.25) * (f[1].pA * f[1].qA) * f[3].qB + T(0.25) * (f[1].qA * (T(1) + f[1].xAb - f[1].xaB)) * f[3].qB + T(0.25) * f[1].xab * (f[3].pA * f[3].qB) + T(0.25) * (f[1].pB * f[1].qA) * (f[3].pA * f[3].qB) + T(0.25) * (f[1].qB * (T(1) + f[1].qA)) * f[3].qA - T(0.25) * f[1].xAb * (f[3].pB * f[3].qA) + T(0.25) * (f[1].pA * f[1].qB) * (f[3].pB * f[3].qA) - T(0.25) * (f[1].pA * f[1].qB) * f[3].qA - T(0.25) * f[1].pA * (f[3].qA * f[3].qB) + T(0.25) * f[1].xAb * (f[3].qA * f[3].qB) + T(0.25) * (f[1].pA * f[1].pB) * (f[3].qA * f[3].qB) + T(0.25) * f[1].xab * f[3].Bsgn + T(0.25) * f[1].Bsgn * f[3].xab - f[1].xab * f[3].xab) * (f[1].r2 * f[3].r2);  // pi2_ijij(1, 3)
    const T v163 = (-T(0.25) * (f[3].qA * f[3].qB) * f[1].pB - T(0.25) * f[3].xab * (f[1].pA * f[1].pB) + T(0.25) * (f[3].qA * f[3].qB) * (f[1].pA * f[1].pB) - T(0.25) * f[3].qA * (f[1].pA * f[1].qB) - T(0.25) * (f[3].pA * f[3].pB) * f[1].xab - T(0.25) * (f[3].qA * f[3].qB) * f[1].xab + T(0.25) * (f[3].pA * f[3].qB) * f[1].xab + T(0.25) * (f[3].pB * f[3].qA) * f[1].xab - T(0.25) * (f[3].pA * f[3].qA) * f[1].qB + T(0.25) * (f[3].qA * (T(1) + f[3].xAb - f[3].xaB)) * f[1].qB + T(0.25) * f[3].xab * (f[1].pA * f[1].qB) + T(0.25) * (f[3].pB * f[3].qA) * (f[1].pA * f[1].qB) + T(0.25) * (f[3].qB * (T(1) + f[3].qA)) * f[1].qA - T(0.25) * f[3].xAb * (f[1].pB * f[1].qA) + T(0.25) * (f[3].pA * f[3].qB) * (f[1].pB * f[1].qA) - T(0.25) * (f[3].pA * f[3].qB) * f[1].qA - T(0.25) * f[3].pA * (f[1].qA * f[1].qB) + T(0.25) * f[3].xAb * (f[1].qA * f[1].qB) + T(0.25) * (f[3].pA * f[3].pB) * (f[1].qA * f[1].qB) + T(0.25) * f[3].xab * f[1].Bsgn + T(0.25) * f[3].Bsgn * f[1].xab - f[3].xab * f[1].xab) * (f[3].r2 * f[1].r2);  // pi2_ijij(3, 1)
    const T v164 = T(0.5) * (f[1].p * f[3].r + f[1].r * f[3].p) * f[2].BR;  // pi2_ijkk(1, 3, 2)
    const T v165 = f[2].BL * T(0.5) * (f[1].q * f[3].s + f[1].s * f[3].q);  // pi2_iikl(2, 1, 3)
    const T v166 = f[1].r * (f[3].C00 * f[2].s + f[3].C01 * f[2].q) + f[1].p * (f[3].C10 * f[2].s + f[3].C11 * f[2].q);  // pi2_shared(3, 1, 2)
    const T v167 = f[2].r * (f[3].C00 * f[1].s + f[3].C01 * f[1].q) + f[2].p * (f[3].C10 * f[1].s + f[3].C11 * f[1].q);  // pi2_shared(3, 2, 1)
    const T v168 = (f[3].BP3 * f[1].pA + f[3].BR3 * f[1].qA) * (f[3].r3 * f[1].r1);  // pi2_ijii(3, 1)
    const T v169 = (f[3].AQ3 * f[1].pB + f[3].AS3 * f[1].qB) * (f[3].r3 * f[1].r1);  // pi2_iiij(3, 1)
    const T v170 = f[2].PI1;  // pi2_same(2,)
    const T v171 = (f[2].AQ3 * f[3].pB + f[2].AS3 * f[3].qB) * (f[2].r3 * f[3].r1);  // pi2_iiij(2, 3)
    const T v172 = (f[2].BP3 * f[3].pA + f[2].BR3 * f[3].qA) * (f[2].r3 * f[3].r1);  // pi2_ijii(2, 3)
    const T v173 = f[2].BL * f[3].BR;  // pi2_iikk(2, 3)
    const T v174 = f[3].BL * f[2].BR;  // pi2_iikk(3, 2)
    const T v175 = (-T(0.25) * (f[2].qA * f[2].qB) * f[3].pB - T(0.25) * f[2].xab * (f[3].pA * f[3].pB) + T(0.25) * (f[2].qA * f[2].qB) * (f[3].pA * f[3].pB) - T(0.25) * f[2].qA * (f[3].pA * f[3].qB) - T(0.25) * (f[2].pA * f[2].pB) * f[3].xab - T(0.25) * (f[2].qA * f[2].qB) * f[3].xab + T(0.25) * (f[2].pA * f[2].qB) * f[3].xab + T(0.25) * (f[2].pB * f[2].qA) * f[3].xab - T(0.25) * (f[2].pA * f[2].qA) * f[3].qB + T(0.25) * (f[2].qA * (T(1) + f[2].xAb - f[2].xaB)) * f[3].qB + T(0.25) * f[2].xab * (f[3].pA * f[3].qB) + T(0.25) * (f[2].pB * f[2].qA) * (f[3].pA * f[3].qB) + T(0.25) * (f[2].qB * (T(1) + f[2].qA)) * f[3].qA - T(0.25) * f[2].xAb * (f[3].pB * f[3].qA) + T(0.25) * (f[2].pA * f[2].qB) * (f[3].pB * f[3].qA) - T(0.25) * (f[2].pA * f[2].qB) * f[3].qA - T(0.25) * f[2].pA * (f[3].qA * f[3].qB) + T(0.25) * f[2].xAb * (f[3].qA * f[3].qB) + T(0.25) * (f[2].pA * f[2].pB) * (f[3].qA * f[3].qB) + T(0.25) * f[2].xab * f[3].Bsgn + T(0.25) * f[2].Bsgn * f[3].xab - f[2].xab * f[3].xab) * (f[2].r2 * f[3].r2);  // pi2_ijij(2, 3)
    const T v176 = (-T(0.25) * (f[3].qA * f[3].qB) * f[2].pB - T(0.25) * f[3].xab * (f[2].pA * f[2].pB) + T(0.25) * (f[3].qA * f[3].qB) * (f[2].pA * f[2].pB) - T(0.25) * f[3].qA * (f[2].pA * f[2].qB) - T(0.25) * (f[3].pA * f[3].pB) * f[2].xab - T(0.25) * (f[3].qA * f[3].qB) * f[2].xab + T(0.25) * (f[3].pA * f[3].qB) * f[2].xab + T(0.25) * (f[3].pB * f[3].qA) * f[2].xab - T(0.25) * (f[3].pA * f[3].qA) * f[2].qB + T(0.25) * (f[3].qA * (T(1) + f[3].xAb - f[3].xaB)) * f[2].qB + T(0.25) * f[3].xab * (f[2].pA * f[2].qB) + T(0.25) * (f[3].pB * f[3].qA) * (f[2].pA * f[2].qB) + T(0.25) * (f[3].qB * (T(1) + f[3].qA)) * f[2].qA - T(0.25) * f[3].xAb * (f[2].pB * f[2].qA) + T(0.25) * (f[3].pA * f[3].qB) * (f[2].pB * f[2].qA) - T(0.25) * (f[3].pA * f[3].qB) * f[2].qA - T(0.25) * f[3].pA * (f[2].qA * f[2].qB) + T(0.25) * f[3].xAb * (f[2].qA * f[2].qB) + T(0.25) * (f[3].pA * f[3].pB) * (f[2].qA * f[2].qB) + T(0.25) * f[3].xab * f[2].Bsgn + T(0.25) * f[3].Bsgn * f[2].xab - f[3].xab * f[2].xab) * (f[3].r2 * f[2].r2);  // pi2_ijij(3, 2)
    const T v177 = (f[3].BP3 * f[2].pA + f[3].BR3 * f[2].qA) * (f[3].r3 * f[2].r1);  // pi2_ijii(3, 2)
    const T v178 = (f[3].AQ3 * f[2].pB + f[3].AS3 * f[2].qB) * (f[3].r3 * f[2].r1);  // pi2_iiij(3, 2)
    const T v179 = f[3].PI1;  // pi2_same(3,)
    acc[0] += v0;  // DD_0_0
    acc[1] += v1;  // DD_0_1
    acc[2] += v2;  // DD_0_2
    acc[3] += v3;  // DD_0_3
    acc[4] += v4;  // DD_1_1
    acc[5] += v5;  // DD_1_2
    acc[6] += v6;  // DD_1_3
    acc[7] += v7;  // DD_2_2
    acc[8] += v8;  // DD_2_3
    acc[9] += v9;  // DD_3_3
    acc[10] += v10;  // Dz_0_0_0
    acc[11] += T(0.5) * (v11 + v12);  // Dz_0_0_1
    acc[12] += T(0.5) * (v13 + v14);  // Dz_0_0_2
    acc[13] += T(0.5) * (v15 + v16);  // Dz_0_0_3
    acc[14] += v17;  // Dz_0_1_1
    acc[15] += T(0.5) * (v18 + v19);  // Dz_0_1_2
    acc[16] += T(0.5) * (v20 + v21);  // Dz_0_1_3
    acc[17] += v22;  // Dz_0_2_2
    acc[18] += T(0.5) * (v23 + v24);  // Dz_0_2_3
    acc[19] += v25;  // Dz_0_3_3
    acc[20] += v26;  // Dz_1_0_0
    acc[21] += T(0.5) * (v27 + v28);  // Dz_1_0_1
    acc[22] += T(0.5) * (v29 + v30);  // Dz_1_0_2
    acc[23] += T(0.5) * (v31 + v32);  // Dz_1_0_3
    acc[24] += v33;  // Dz_1_1_1
    acc[25] += T(0.5) * (v34 + v35);  // Dz_1_1_2
    acc[26] += T(0.5) * (v36 + v37);  // Dz_1_1_3
    acc[27] += v38;  // Dz_1_2_2
    acc[28] += T(0.5) * (v39 + v40);  // Dz_1_2_3
    acc[29] += v41;  // Dz_1_3_3
    acc[30] += v42;  // Dz_2_0_0
    acc[31] += T(0.5) * (v43 + v44);  // Dz_2_0_1
    acc[32] += T(0.5) * (v45 + v46);  // Dz_2_0_2
    acc[33] += T(0.5) * (v47 + v48);  // Dz_2_0_3
    acc[34] += v49;  // Dz_2_1_1
    acc[35] += T(0.5) * (v50 + v51);  // Dz_2_1_2
    acc[36] += T(0.5) * (v52 + v53);  // Dz_2_1_3
    acc[37] += v54;  // Dz_2_2_2
    acc[38] += T(0.5) * (v55 + v56);  // Dz_2_2_3
    acc[39] += v57;  // Dz_2_3_3
    acc[40] += v58;  // Dz_3_0_0
    acc[41] += T(0.5) * (v59 + v60);  // Dz_3_0_1
    acc[42] += T(0.5) * (v61 + v62);  // Dz_3_0_2
    acc[43] += T(0.5) * (v63 + v64);  // Dz_3_0_3
    acc[44] += v65;  // Dz_3_1_1
    acc[45] += T(0.5) * (v66 + v67);  // Dz_3_1_2
    acc[46] += T(0.5) * (v68 + v69);  // Dz_3_1_3
    acc[47] += v70;  // Dz_3_2_2
    acc[48] += T(0.5) * (v71 + v72);  // Dz_3_2_3
    acc[49] += v73;  // Dz_3_3_3
    acc[50] += v74;  // pi2_0_0_0_0
    acc[51] += T(0.5) * (v75 + v76);  // pi2_0_0_0_1
    acc[52] += T(0.5) * (v77 + v78);  // pi2_0_0_0_2
    acc[53] += T(0.5) * (v79 + v80);  // pi2_0_0_0_3
    acc[54] += T(0.5) * (v81 + v82);  // pi2_0_0_1_1
    acc[55] += T(0.5) * (v83 + v84);  // pi2_0_0_1_2
    acc[56] += T(0.5) * (v85 + v86);  // pi2_0_0_1_3
    acc[57] += T(0.5) * (v87 + v88);  // pi2_0_0_2_2
    acc[58] += T(0.5) * (v89 + v90);  // pi2_0_0_2_3
    acc[59] += T(0.5) * (v91 + v92);  // pi2_0_0_3_3
    acc[60] += T(0.5) * (v93 + v94);  // pi2_0_1_0_1
    acc[61] += T(0.5) * (v95 + v96);  // pi2_0_1_0_2
    acc[62] += T(0.5) * (v97 + v98);  // pi2_0_1_0_3
    acc[63] += T(0.5) * (v99 + v100);  // pi2_0_1_1_1
    acc[64] += T(0.5) * (v101 + v102);  // pi2_0_1_1_2
    acc[65] += T(0.5) * (v103 + v104);  // pi2_0_1_1_3
    acc[66] += T(0.5) * (v105 + v106);  // pi2_0_1_2_2
    acc[67] += T(0.5) * (v107 + v108);  // pi2_0_1_2_3
    acc[68] += T(0.5) * (v109 + v110);  // pi2_0_1_3_3
    acc[69] += T(0.5) * (v111 + v112);  // pi2_0_2_0_2
    acc[70] += T(0.5) * (v113 + v114);  // pi2_0_2_0_3
    acc[71] += T(0.5) * (v115 + v116);  // pi2_0_2_1_1
    acc[72] += T(0.5) * (v117 + v118);  // pi2_0_2_1_2
    acc[73] += T(0.5) * (v119 + v120);  // pi2_0_2_1_3
    acc[74] += T(0.5) * (v121 + v122);  // pi2_0_2_2_2
    acc[75] += T(0.5) * (v123 + v124);  // pi2_0_2_2_3
    acc[76] += T(0.5) * (v125 + v126);  // pi2_0_2_3_3
    acc[77] += T(0.5) * (v127 + v128);  // pi2_0_3_0_3
    acc[78] += T(0.5) * (v129 + v130);  // pi2_0_3_1_1
    acc[79] += T(0.5) * (v131 + v132);  // pi2_0_3_1_2
    acc[80] += T(0.5) * (v133 + v134);  // pi2_0_3_1_3
    acc[81] += T(0.5) * (v135 + v136);  // pi2_0_3_2_2
    acc[82] += T(0.5) * (v137 + v138);  // pi2_0_3_2_3
    acc[83] += T(0.5) * (v139 + v140);  // pi2_0_3_3_3
    acc[84] += v141;  // pi2_1_1_1_1
    acc[85] += T(0.5) * (v142 + v143);  // pi2_1_1_1_2
    acc[86] += T(0.5) * (v144 + v145);  // pi2_1_1_1_3
    acc[87] += T(0.5) * (v146 + v147);  // pi2_1_1_2_2
    acc[88] += T(0.5) * (v148 + v149);  // pi2_1_1_2_3
    acc[89] += T(0.5) * (v150 + v151);  // pi2_1_1_3_3
    acc[90] += T(0.5) * (v152 + v153);  // pi2_1_2_1_2
    acc[91] += T(0.5) * (v154 + v155);  // pi2_1_2_1_3
    acc[92] += T(0.5) * (v156 + v157);  // pi2_1_2_2_2
    acc[93] += T(0.5) * (v158 + v159);  // pi2_1_2_2_3
    acc[94] += T(0.5) * (v160 + v161);  // pi2_1_2_3_3
    acc[95] += T(0.5) * (v162 + v163);  // pi2_1_3_1_3
    acc[96] += T(0.5) * (v164 + v165);  // pi2_1_3_2_2
    acc[97] += T(0.5) * (v166 + v167);  // pi2_1_3_2_3
    acc[98] += T(0.5) * (v168 + v169);  // pi2_1_3_3_3
    acc[99] += v170;  // pi2_2_2_2_2
    acc[100] += T(0.5) * (v171 + v172);  // pi2_2_2_2_3
    acc[101] += T(0.5) * (v173 + v174);  // pi2_2_2_3_3
    acc[102] += T(0.5) * (v175 + v176);  // pi2_2_3_2_3
    acc[103] += T(0.5) * (v177 + v178);  // pi2_2_3_3_3
    acc[104] += v179;  // pi2_3_3_3_3
}

template <typename T>
LDK_DEV T hap_raw_by_case(int case_id, const int* g, const HapFeat<T>* f) {
    switch (case_id) {
    case 0: return f[g[0]].DDs * f[g[0]].r4;  // dd1
    case 1: return (f[g[0]].E * f[g[1]].E) * (f[g[0]].r2 * f[g[1]].r2);  // dd2
    case 2: return f[g[0]].DZs * f[g[0]].r4;  // dz_iii
    case 3: return (f[g[0]].a * f[g[0]].E * f[g[1]].b) * (f[g[0]].r3 * f[g[1]].r1);  // dz_iij
    case 4: return (f[g[0]].b * f[g[0]].E * f[g[1]].a) * (f[g[0]].r3 * f[g[1]].r1);  // dz_iji
    case 5: return (f[g[0]].E * (f[g[1]].s + f[g[1]].b * f[g[1]].a)) * (f[g[0]].r2 * f[g[1]].r2);  // dz_ijj
    case 6: return (f[g[0]].E * f[g[1]].a * f[g[2]].b) * (f[g[0]].r2 * f[g[1]].r1 * f[g[2]].r1);  // dz_ijk
    case 7: return f[g[0]].PIs * f[g[0]].r4;  // pi2_same
    case 8: return (f[g[0]].fA * f[g[1]].fB) * (f[g[0]].r2 * f[g[1]].r2);  // pi2_iikk
    case 9: return T(0.5) * (f[g[0]].fA * (f[g[1]].pB * f[g[2]].qB + f[g[1]].qB * f[g[2]].pB)) * (f[g[0]].r2 * f[g[1]].r1 * f[g[2]].r1);  // pi2_iikl
    case 10: return T(0.5) * (f[g[2]].fB * (f[g[0]].pA * f[g[1]].qA + f[g[0]].qA * f[g[1]].pA)) * (f[g[2]].r2 * f[g[0]].r1 * f[g[1]].r1);  // pi2_ijkk
    case 11: return T(0.25) * ((f[g[0]].pA * f[g[1]].qA + f[g[0]].qA * f[g[1]].pA) * (f[g[2]].pB * f[g[3]].qB + f[g[2]].qB * f[g[3]].pB)) * (f[g[0]].r1 * f[g[1]].r1 * f[g[2]].r1 * f[g[3]].r1);  // pi2_alldiff
    case 12: return T(0.5) * (f[g[1]].pB * f[g[0]].T1 + f[g[1]].qB * f[g[0]].T2) * (f[g[0]].r3 * f[g[1]].r1);  // pi2_triple
    case 13: return T(0.25) * ((f[g[0]].pA * f[g[1]].qA + f[g[0]].qA * f[g[1]].pA) * (f[g[0]].pB * f[g[1]].qB + f[g[0]].qB * f[g[1]].pB) + (f[g[0]].Q1 * f[g[1]].c4 + f[g[0]].Q2 * f[g[1]].c3 + f[g[0]].Q3 * f[g[1]].c2 + f[g[0]].Q4 * f[g[1]].c1 - (f[g[0]].c1 * f[g[1]].L1 + f[g[0]].c2 * f[g[1]].L2 + f[g[0]].c3 * f[g[1]].L3 + f[g[0]].c4 * f[g[1]].L4))) * (f[g[0]].r2 * f[g[1]].r2);  // pi2_ijij
    case 14: return T(0.25) * (f[g[1]].pA * (f[g[2]].pB * (f[g[0]].L1 - f[g[0]].c4) + f[g[2]].qB * (f[g[0]].L2 - f[g[0]].c3)) + f[g[1]].qA * (f[g[2]].pB * (f[g[0]].L3 - f[g[0]].c2) + f[g[2]].qB * (f[g[0]].L4 - f[g[0]].c1))) * (f[g[0]].r2 * f[g[1]].r1 * f[g[2]].r1);  // pi2_shared
    default: return T(0);
    }
}

template <int P> struct HapNStats;
template <> struct HapNStats<1> { static constexpr int value = 3; };
template <> struct HapNStats<2> { static constexpr int value = 15; };
template <> struct HapNStats<3> { static constexpr int value = 45; };
template <> struct HapNStats<4> { static constexpr int value = 105; };

template <typename T, int P>
LDK_DEV void hap_features(HapFeat<T>& x) {
    if constexpr (P == 1) hap_features_P1<T>(x);
    else if constexpr (P == 2) hap_features_P2<T>(x);
    else if constexpr (P == 3) hap_features_P3<T>(x);
    else hap_features_P4<T>(x);
}
template <typename T, int P>
LDK_DEV void geno_features(GenoFeat<T>& x) {
    if constexpr (P == 1) geno_features_P1<T>(x);
    else if constexpr (P == 2) geno_features_P2<T>(x);
    else if constexpr (P == 3) geno_features_P3<T>(x);
    else geno_features_P4<T>(x);
}
template <typename T, int P>
LDK_DEV void geno_stats(const GenoFeat<T>* f, T* acc) {
    if constexpr (P == 1) geno_stats_P1<T>(f, acc);
    else if constexpr (P == 2) geno_stats_P2<T>(f, acc);
    else if constexpr (P == 3) geno_stats_P3<T>(f, acc);
    else geno_stats_P4<T>(f, acc);
}
template <typename T, int P>
LDK_DEV void hap_stats(const HapFeat<T>* f, T* acc) {
    if constexpr (P == 1) hap_stats_P1<T>(f, acc);
    else if constexpr (P == 2) hap_stats_P2<T>(f, acc);
    else if constexpr (P == 3) hap_stats_P3<T>(f, acc);
    else hap_stats_P4<T>(f, acc);
}
