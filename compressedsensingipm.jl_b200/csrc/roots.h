// Roots of unity W_R^m = exp(-2*pi*i*m/R) for the composite register
// butterflies, as correctly rounded double literals (generated from a
// 60-digit decimal evaluation; the tables of 18, 24, 27 and 30 by
// gen_roots.py, which reproduces the others bit for bit except that it
// writes exact zeros at multiples of pi/2).  Each function folds to a
// constant when m is a compile-time value.
#pragma once

namespace csipm {

__device__ __forceinline__ constexpr double root_re6(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.5;
        case 2: return -0.5;
        case 3: return -1.0;
        case 4: return -0.5;
        case 5: return 0.5;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im6(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.8660254037844386;
        case 2: return -0.8660254037844386;
        case 3: return -1.4628678077038063e-59;
        case 4: return 0.8660254037844386;
        case 5: return 0.8660254037844386;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re9(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.766044443118978;
        case 2: return 0.17364817766693036;
        case 3: return -0.5;
        case 4: return -0.9396926207859084;
        case 5: return -0.9396926207859084;
        case 6: return -0.5;
        case 7: return 0.17364817766693036;
        case 8: return 0.766044443118978;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im9(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.6427876096865394;
        case 2: return -0.984807753012208;
        case 3: return -0.8660254037844386;
        case 4: return -0.3420201433256687;
        case 5: return 0.3420201433256687;
        case 6: return 0.8660254037844386;
        case 7: return 0.984807753012208;
        case 8: return 0.6427876096865394;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re10(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.8090169943749475;
        case 2: return 0.30901699437494745;
        case 3: return -0.30901699437494745;
        case 4: return -0.8090169943749475;
        case 5: return -1.0;
        case 6: return -0.8090169943749475;
        case 7: return -0.30901699437494745;
        case 8: return 0.30901699437494745;
        case 9: return 0.8090169943749475;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im10(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.5877852522924731;
        case 2: return -0.9510565162951535;
        case 3: return -0.9510565162951535;
        case 4: return -0.5877852522924731;
        case 5: return -4.582863744331626e-60;
        case 6: return 0.5877852522924731;
        case 7: return 0.9510565162951535;
        case 8: return 0.9510565162951535;
        case 9: return 0.5877852522924731;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re12(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.8660254037844386;
        case 2: return 0.5;
        case 3: return 2.3545201566946508e-60;
        case 4: return -0.5;
        case 5: return -0.8660254037844386;
        case 6: return -1.0;
        case 7: return -0.8660254037844386;
        case 8: return -0.5;
        case 9: return -8.32451261776133e-60;
        case 10: return 0.5;
        case 11: return 0.8660254037844386;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im12(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.5;
        case 2: return -0.8660254037844386;
        case 3: return -1.0;
        case 4: return -0.8660254037844386;
        case 5: return -0.5;
        case 6: return -4.582863744331626e-60;
        case 7: return 0.5;
        case 8: return 0.8660254037844386;
        case 9: return 1.0;
        case 10: return 0.8660254037844386;
        case 11: return 0.5;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re15(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9135454576426009;
        case 2: return 0.6691306063588582;
        case 3: return 0.30901699437494745;
        case 4: return -0.10452846326765347;
        case 5: return -0.5;
        case 6: return -0.8090169943749475;
        case 7: return -0.9781476007338057;
        case 8: return -0.9781476007338057;
        case 9: return -0.8090169943749475;
        case 10: return -0.5;
        case 11: return -0.10452846326765347;
        case 12: return 0.30901699437494745;
        case 13: return 0.6691306063588582;
        case 14: return 0.9135454576426009;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im15(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.4067366430758002;
        case 2: return -0.7431448254773942;
        case 3: return -0.9510565162951535;
        case 4: return -0.9945218953682733;
        case 5: return -0.8660254037844386;
        case 6: return -0.5877852522924731;
        case 7: return -0.20791169081775934;
        case 8: return 0.20791169081775934;
        case 9: return 0.5877852522924731;
        case 10: return 0.8660254037844386;
        case 11: return 0.9945218953682733;
        case 12: return 0.9510565162951535;
        case 13: return 0.7431448254773942;
        case 14: return 0.4067366430758002;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re16(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9238795325112867;
        case 2: return 0.7071067811865476;
        case 3: return 0.3826834323650898;
        case 4: return 2.3545201566946508e-60;
        case 5: return -0.3826834323650898;
        case 6: return -0.7071067811865476;
        case 7: return -0.9238795325112867;
        case 8: return -1.0;
        case 9: return -0.9238795325112867;
        case 10: return -0.7071067811865476;
        case 11: return -0.3826834323650898;
        case 12: return -8.32451261776133e-60;
        case 13: return 0.3826834323650898;
        case 14: return 0.7071067811865476;
        case 15: return 0.9238795325112867;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im16(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.3826834323650898;
        case 2: return -0.7071067811865476;
        case 3: return -0.9238795325112867;
        case 4: return -1.0;
        case 5: return -0.9238795325112867;
        case 6: return -0.7071067811865476;
        case 7: return -0.3826834323650898;
        case 8: return -4.582863744331626e-60;
        case 9: return 0.3826834323650898;
        case 10: return 0.7071067811865476;
        case 11: return 0.9238795325112867;
        case 12: return 1.0;
        case 13: return 0.9238795325112867;
        case 14: return 0.7071067811865476;
        case 15: return 0.3826834323650898;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re20(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9510565162951535;
        case 2: return 0.8090169943749475;
        case 3: return 0.5877852522924731;
        case 4: return 0.30901699437494745;
        case 5: return 2.3545201566946508e-60;
        case 6: return -0.30901699437494745;
        case 7: return -0.5877852522924731;
        case 8: return -0.8090169943749475;
        case 9: return -0.9510565162951535;
        case 10: return -1.0;
        case 11: return -0.9510565162951535;
        case 12: return -0.8090169943749475;
        case 13: return -0.5877852522924731;
        case 14: return -0.30901699437494745;
        case 15: return -8.32451261776133e-60;
        case 16: return 0.30901699437494745;
        case 17: return 0.5877852522924731;
        case 18: return 0.8090169943749475;
        case 19: return 0.9510565162951535;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im20(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.30901699437494745;
        case 2: return -0.5877852522924731;
        case 3: return -0.8090169943749475;
        case 4: return -0.9510565162951535;
        case 5: return -1.0;
        case 6: return -0.9510565162951535;
        case 7: return -0.8090169943749475;
        case 8: return -0.5877852522924731;
        case 9: return -0.30901699437494745;
        case 10: return -4.582863744331626e-60;
        case 11: return 0.30901699437494745;
        case 12: return 0.5877852522924731;
        case 13: return 0.8090169943749475;
        case 14: return 0.9510565162951535;
        case 15: return 1.0;
        case 16: return 0.9510565162951535;
        case 17: return 0.8090169943749475;
        case 18: return 0.5877852522924731;
        case 19: return 0.30901699437494745;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re25(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9685831611286311;
        case 2: return 0.8763066800438636;
        case 3: return 0.7289686274214116;
        case 4: return 0.5358267949789967;
        case 5: return 0.30901699437494745;
        case 6: return 0.06279051952931337;
        case 7: return -0.18738131458572463;
        case 8: return -0.42577929156507266;
        case 9: return -0.6374239897486897;
        case 10: return -0.8090169943749475;
        case 11: return -0.9297764858882515;
        case 12: return -0.9921147013144779;
        case 13: return -0.9921147013144779;
        case 14: return -0.9297764858882515;
        case 15: return -0.8090169943749475;
        case 16: return -0.6374239897486897;
        case 17: return -0.42577929156507266;
        case 18: return -0.18738131458572463;
        case 19: return 0.06279051952931337;
        case 20: return 0.30901699437494745;
        case 21: return 0.5358267949789967;
        case 22: return 0.7289686274214116;
        case 23: return 0.8763066800438636;
        case 24: return 0.9685831611286311;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im25(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.2486898871648548;
        case 2: return -0.48175367410171527;
        case 3: return -0.6845471059286887;
        case 4: return -0.8443279255020151;
        case 5: return -0.9510565162951535;
        case 6: return -0.9980267284282716;
        case 7: return -0.9822872507286887;
        case 8: return -0.9048270524660196;
        case 9: return -0.7705132427757893;
        case 10: return -0.5877852522924731;
        case 11: return -0.368124552684678;
        case 12: return -0.12533323356430426;
        case 13: return 0.12533323356430426;
        case 14: return 0.368124552684678;
        case 15: return 0.5877852522924731;
        case 16: return 0.7705132427757893;
        case 17: return 0.9048270524660196;
        case 18: return 0.9822872507286887;
        case 19: return 0.9980267284282716;
        case 20: return 0.9510565162951535;
        case 21: return 0.8443279255020151;
        case 22: return 0.6845471059286887;
        case 23: return 0.48175367410171527;
        case 24: return 0.2486898871648548;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re32(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9807852804032304;
        case 2: return 0.9238795325112867;
        case 3: return 0.8314696123025452;
        case 4: return 0.7071067811865476;
        case 5: return 0.5555702330196022;
        case 6: return 0.3826834323650898;
        case 7: return 0.19509032201612828;
        case 8: return 2.3545201566946508e-60;
        case 9: return -0.19509032201612828;
        case 10: return -0.3826834323650898;
        case 11: return -0.5555702330196022;
        case 12: return -0.7071067811865476;
        case 13: return -0.8314696123025452;
        case 14: return -0.9238795325112867;
        case 15: return -0.9807852804032304;
        case 16: return -1.0;
        case 17: return -0.9807852804032304;
        case 18: return -0.9238795325112867;
        case 19: return -0.8314696123025452;
        case 20: return -0.7071067811865476;
        case 21: return -0.5555702330196022;
        case 22: return -0.3826834323650898;
        case 23: return -0.19509032201612828;
        case 24: return -8.32451261776133e-60;
        case 25: return 0.19509032201612828;
        case 26: return 0.3826834323650898;
        case 27: return 0.5555702330196022;
        case 28: return 0.7071067811865476;
        case 29: return 0.8314696123025452;
        case 30: return 0.9238795325112867;
        case 31: return 0.9807852804032304;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im32(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.19509032201612828;
        case 2: return -0.3826834323650898;
        case 3: return -0.5555702330196022;
        case 4: return -0.7071067811865476;
        case 5: return -0.8314696123025452;
        case 6: return -0.9238795325112867;
        case 7: return -0.9807852804032304;
        case 8: return -1.0;
        case 9: return -0.9807852804032304;
        case 10: return -0.9238795325112867;
        case 11: return -0.8314696123025452;
        case 12: return -0.7071067811865476;
        case 13: return -0.5555702330196022;
        case 14: return -0.3826834323650898;
        case 15: return -0.19509032201612828;
        case 16: return -4.582863744331626e-60;
        case 17: return 0.19509032201612828;
        case 18: return 0.3826834323650898;
        case 19: return 0.5555702330196022;
        case 20: return 0.7071067811865476;
        case 21: return 0.8314696123025452;
        case 22: return 0.9238795325112867;
        case 23: return 0.9807852804032304;
        case 24: return 1.0;
        case 25: return 0.9807852804032304;
        case 26: return 0.9238795325112867;
        case 27: return 0.8314696123025452;
        case 28: return 0.7071067811865476;
        case 29: return 0.5555702330196022;
        case 30: return 0.3826834323650898;
        case 31: return 0.19509032201612828;
        default: return 0.0;
    }
}

__device__ __forceinline__ constexpr double root_re18(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9396926207859084;
        case 2: return 0.766044443118978;
        case 3: return 0.5;
        case 4: return 0.17364817766693036;
        case 5: return -0.17364817766693036;
        case 6: return -0.5;
        case 7: return -0.766044443118978;
        case 8: return -0.9396926207859084;
        case 9: return -1.0;
        case 10: return -0.9396926207859084;
        case 11: return -0.766044443118978;
        case 12: return -0.5;
        case 13: return -0.17364817766693036;
        case 14: return 0.17364817766693036;
        case 15: return 0.5;
        case 16: return 0.766044443118978;
        case 17: return 0.9396926207859084;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im18(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.3420201433256687;
        case 2: return -0.6427876096865394;
        case 3: return -0.8660254037844386;
        case 4: return -0.984807753012208;
        case 5: return -0.984807753012208;
        case 6: return -0.8660254037844386;
        case 7: return -0.6427876096865394;
        case 8: return -0.3420201433256687;
        case 9: return 0.0;
        case 10: return 0.3420201433256687;
        case 11: return 0.6427876096865394;
        case 12: return 0.8660254037844386;
        case 13: return 0.984807753012208;
        case 14: return 0.984807753012208;
        case 15: return 0.8660254037844386;
        case 16: return 0.6427876096865394;
        case 17: return 0.3420201433256687;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re24(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9659258262890683;
        case 2: return 0.8660254037844386;
        case 3: return 0.7071067811865476;
        case 4: return 0.5;
        case 5: return 0.25881904510252074;
        case 6: return 0.0;
        case 7: return -0.25881904510252074;
        case 8: return -0.5;
        case 9: return -0.7071067811865476;
        case 10: return -0.8660254037844386;
        case 11: return -0.9659258262890683;
        case 12: return -1.0;
        case 13: return -0.9659258262890683;
        case 14: return -0.8660254037844386;
        case 15: return -0.7071067811865476;
        case 16: return -0.5;
        case 17: return -0.25881904510252074;
        case 18: return 0.0;
        case 19: return 0.25881904510252074;
        case 20: return 0.5;
        case 21: return 0.7071067811865476;
        case 22: return 0.8660254037844386;
        case 23: return 0.9659258262890683;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im24(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.25881904510252074;
        case 2: return -0.5;
        case 3: return -0.7071067811865476;
        case 4: return -0.8660254037844386;
        case 5: return -0.9659258262890683;
        case 6: return -1.0;
        case 7: return -0.9659258262890683;
        case 8: return -0.8660254037844386;
        case 9: return -0.7071067811865476;
        case 10: return -0.5;
        case 11: return -0.25881904510252074;
        case 12: return 0.0;
        case 13: return 0.25881904510252074;
        case 14: return 0.5;
        case 15: return 0.7071067811865476;
        case 16: return 0.8660254037844386;
        case 17: return 0.9659258262890683;
        case 18: return 1.0;
        case 19: return 0.9659258262890683;
        case 20: return 0.8660254037844386;
        case 21: return 0.7071067811865476;
        case 22: return 0.5;
        case 23: return 0.25881904510252074;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re27(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9730448705798238;
        case 2: return 0.8936326403234123;
        case 3: return 0.766044443118978;
        case 4: return 0.5971585917027862;
        case 5: return 0.39607976603915684;
        case 6: return 0.17364817766693036;
        case 7: return -0.05814482891047583;
        case 8: return -0.28680323271109026;
        case 9: return -0.5;
        case 10: return -0.6862416378687336;
        case 11: return -0.8354878114129364;
        case 12: return -0.9396926207859084;
        case 13: return -0.993238357741943;
        case 14: return -0.993238357741943;
        case 15: return -0.9396926207859084;
        case 16: return -0.8354878114129364;
        case 17: return -0.6862416378687336;
        case 18: return -0.5;
        case 19: return -0.28680323271109026;
        case 20: return -0.05814482891047583;
        case 21: return 0.17364817766693036;
        case 22: return 0.39607976603915684;
        case 23: return 0.5971585917027862;
        case 24: return 0.766044443118978;
        case 25: return 0.8936326403234123;
        case 26: return 0.9730448705798238;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im27(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.23061587074244017;
        case 2: return -0.44879918020046217;
        case 3: return -0.6427876096865394;
        case 4: return -0.8021231927550437;
        case 5: return -0.918216106880274;
        case 6: return -0.984807753012208;
        case 7: return -0.9983081582712682;
        case 8: return -0.9579895123154889;
        case 9: return -0.8660254037844386;
        case 10: return -0.7273736415730487;
        case 11: return -0.549508978070806;
        case 12: return -0.3420201433256687;
        case 13: return -0.11609291412523023;
        case 14: return 0.11609291412523023;
        case 15: return 0.3420201433256687;
        case 16: return 0.549508978070806;
        case 17: return 0.7273736415730487;
        case 18: return 0.8660254037844386;
        case 19: return 0.9579895123154889;
        case 20: return 0.9983081582712682;
        case 21: return 0.984807753012208;
        case 22: return 0.918216106880274;
        case 23: return 0.8021231927550437;
        case 24: return 0.6427876096865394;
        case 25: return 0.44879918020046217;
        case 26: return 0.23061587074244017;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_re30(int m) {
    switch (m) {
        case 0: return 1.0;
        case 1: return 0.9781476007338057;
        case 2: return 0.9135454576426009;
        case 3: return 0.8090169943749475;
        case 4: return 0.6691306063588582;
        case 5: return 0.5;
        case 6: return 0.30901699437494745;
        case 7: return 0.10452846326765347;
        case 8: return -0.10452846326765347;
        case 9: return -0.30901699437494745;
        case 10: return -0.5;
        case 11: return -0.6691306063588582;
        case 12: return -0.8090169943749475;
        case 13: return -0.9135454576426009;
        case 14: return -0.9781476007338057;
        case 15: return -1.0;
        case 16: return -0.9781476007338057;
        case 17: return -0.9135454576426009;
        case 18: return -0.8090169943749475;
        case 19: return -0.6691306063588582;
        case 20: return -0.5;
        case 21: return -0.30901699437494745;
        case 22: return -0.10452846326765347;
        case 23: return 0.10452846326765347;
        case 24: return 0.30901699437494745;
        case 25: return 0.5;
        case 26: return 0.6691306063588582;
        case 27: return 0.8090169943749475;
        case 28: return 0.9135454576426009;
        case 29: return 0.9781476007338057;
        default: return 0.0;
    }
}
__device__ __forceinline__ constexpr double root_im30(int m) {
    switch (m) {
        case 0: return -0.0;
        case 1: return -0.20791169081775934;
        case 2: return -0.4067366430758002;
        case 3: return -0.5877852522924731;
        case 4: return -0.7431448254773942;
        case 5: return -0.8660254037844386;
        case 6: return -0.9510565162951535;
        case 7: return -0.9945218953682733;
        case 8: return -0.9945218953682733;
        case 9: return -0.9510565162951535;
        case 10: return -0.8660254037844386;
        case 11: return -0.7431448254773942;
        case 12: return -0.5877852522924731;
        case 13: return -0.4067366430758002;
        case 14: return -0.20791169081775934;
        case 15: return 0.0;
        case 16: return 0.20791169081775934;
        case 17: return 0.4067366430758002;
        case 18: return 0.5877852522924731;
        case 19: return 0.7431448254773942;
        case 20: return 0.8660254037844386;
        case 21: return 0.9510565162951535;
        case 22: return 0.9945218953682733;
        case 23: return 0.9945218953682733;
        case 24: return 0.9510565162951535;
        case 25: return 0.8660254037844386;
        case 26: return 0.7431448254773942;
        case 27: return 0.5877852522924731;
        case 28: return 0.4067366430758002;
        case 29: return 0.20791169081775934;
        default: return 0.0;
    }
}

template <int R> struct RootTab;
template <> struct RootTab<6> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re6(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im6(m); }
};
template <> struct RootTab<9> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re9(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im9(m); }
};
template <> struct RootTab<10> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re10(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im10(m); }
};
template <> struct RootTab<12> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re12(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im12(m); }
};
template <> struct RootTab<15> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re15(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im15(m); }
};
template <> struct RootTab<16> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re16(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im16(m); }
};
template <> struct RootTab<20> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re20(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im20(m); }
};
template <> struct RootTab<25> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re25(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im25(m); }
};
template <> struct RootTab<32> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re32(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im32(m); }
};

template <> struct RootTab<18> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re18(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im18(m); }
};
template <> struct RootTab<24> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re24(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im24(m); }
};
template <> struct RootTab<27> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re27(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im27(m); }
};
template <> struct RootTab<30> {
    __device__ __forceinline__ static constexpr double re(int m) { return root_re30(m); }
    __device__ __forceinline__ static constexpr double im(int m) { return root_im30(m); }
};

}  // namespace csipm
