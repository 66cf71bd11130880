// TEST INFRASTRUCTURE ONLY. The three SYCL math names the reference's host oracle headers use
// (examples/ns-residual/physics.hpp: sycl::sqrt, sycl::sin, sycl::cos), mapped to the C++ library, so that those
// headers compile as plain C++ for the oracle wrapper (ref_wrap.cpp).
#pragma once
#include <cmath>
namespace sycl { using std::sqrt; using std::sin; using std::cos; }
