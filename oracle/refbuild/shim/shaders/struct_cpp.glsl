/* Case-correcting forwarder: src/Renderer/BVHBuilder.cpp:11 includes
 * "shaders/struct_cpp.glsl" while the directory is "Shaders". TEST INFRASTRUCTURE ONLY. */
#include "Shaders/struct_cpp.glsl"
