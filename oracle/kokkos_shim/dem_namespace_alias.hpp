// Test infrastructure: the reference's broadphase unit test (tests/arborx/test_broadphase_arborx.cpp)
// names the headers' namespace `dem`; the headers define `peclet::dem`. Force-included when that
// test is compiled, so the test source stays unmodified.
#pragma once
namespace peclet {
namespace dem {}
}  // namespace peclet
namespace dem = peclet::dem;
