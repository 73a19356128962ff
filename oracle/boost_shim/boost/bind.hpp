// Test infrastructure: boost::bind / boost::ref over std::bind / std::ref,
// for the reference's host code (all arguments bound, no placeholders).
#pragma once
#include <functional>
namespace boost {
using std::bind;
using std::ref;
}
