// Identity of this plugin SDK.  A plugin records the identity it was compiled
// with, and the library loads only plugins of its own SDK: the interface
// passes C++ objects (std::string, std::vector, std::variant, virtual calls)
// across the library boundary, so both sides must see the same definitions.
#pragma once
#define CUDA_MOEA_NATIVE_BUILD_ID "moea-b200-native-sdk-1"
