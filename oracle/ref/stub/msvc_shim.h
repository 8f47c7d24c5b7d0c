// Force-included when compiling the reference: it names std::sinf / std::cosf, which only
// MSVC's <cmath> declares.
#pragma once
#include <cmath>
namespace std { using ::sinf; using ::cosf; }
