// ref_plugin_adapter.cpp — compiles ONE MSL model plugin (given by the macro
// REF_PLUGIN_SOURCE, e.g. the reference's shaders/test_user_dynamics.metal)
// as C++ and hands its three callables to ref_harness.cpp as untyped
// pointers.  The reference links callables by name through visible function
// tables (src/metal_backend.mm:295-334, 397-439); the harness does the same
// with plain function pointers.  TEST INFRASTRUCTURE ONLY.
#include <metal_stdlib>

#include REF_PLUGIN_SOURCE

extern "C" void* ref_plugin_dynamics() { return reinterpret_cast<void*>(&mppi_dynamics); }
extern "C" void* ref_plugin_stage_cost() { return reinterpret_cast<void*>(&mppi_stage_cost); }
extern "C" void* ref_plugin_terminal_cost() { return reinterpret_cast<void*>(&mppi_terminal_cost); }
