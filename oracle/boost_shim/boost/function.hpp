// Test infrastructure: the part of boost::function the reference's host code
// uses, over std::function (builds the reference's host flow for the
// oracle; no Boost in this image).
#pragma once
#include <functional>
namespace boost {
template <class Sig> using function = std::function<Sig>;
}
