// Empty stand-in for <boost/integer_fwd.hpp>. The reference's
// pairhmm/inter/simd_traits_avx512.h includes it but uses nothing from it;
// Boost is not installed in this image.
#pragma once
