// The peak record of mcstar-libs common/maximum_struct.hpp:3-6, kept bit-compatible:
// pfc_findpeaks writes records of exactly this layout (grid indices stored in T).
#pragma once

template <typename T> struct Maximum {
    T i0, i1, i2;
    float field;
};
