// Symbol visibility for the C-ABI: every library here is built with
// -fvisibility=hidden and exports only what carries NB_API.
#pragma once
#define NB_API extern "C" __attribute__((visibility("default")))
