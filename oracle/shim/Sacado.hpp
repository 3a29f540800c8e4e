// Stand-in for Trilinos' Sacado header, used only to compile the reference's
// LPS kernels for the CPU oracle. The reference instantiates its kernels for
// Sacado::Fad::DFad<double>; here that type is long double, which keeps the
// second explicit instantiation a distinct, compilable type. Nothing in the
// oracle calls the long double instantiation.
#pragma once
#include <cmath>
namespace Sacado { namespace Fad { template <typename T> using DFad = long double; } }
