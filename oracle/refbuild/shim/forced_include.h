/* oracle/refbuild/shim/forced_include.h -- TEST INFRASTRUCTURE ONLY.
 * Standard headers the reference's MSVC build pulls in transitively, plus the
 * Windows `byte` typedef its sources use (src/Renderer/BVHBuilder.cpp:1471). */
#pragma once
#include <functional>
#include <memory>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <cstring>
#include <chrono>
#include <iostream>
typedef unsigned char byte;
