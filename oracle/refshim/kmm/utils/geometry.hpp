// Host stand-in for the one kmm geometry type the compas-toolkit kernel headers name.
// TEST INFRASTRUCTURE ONLY (oracle/ref_sim.cpp); kmm itself is an empty submodule in the
// reference tree and is not reproduced here.
#pragma once

namespace kmm {
template<typename T>
struct Range {
    T begin = 0, end = 0;
    T size() const { return end - begin; }
};
}  // namespace kmm
