// Test library registered with another SDK's build id: the host must refuse it
// before touching any C++ object of the registration.
#include <cstdint>

struct Prefix {
    std::uint32_t abi;
    const char* build_id;
};

extern "C" __attribute__((visibility("default"))) const Prefix* cuda_moea_problem_v1()
{
    static const Prefix p{1, "some-other-sdk"};
    return &p;
}
