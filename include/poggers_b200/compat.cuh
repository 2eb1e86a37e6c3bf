// compat.cuh -- source compatibility for code written against the reference.
//
// A translation unit that used
//     #include <poggers/data_structs/tcf.cuh>            (or any table header)
//     using T = poggers::tables::static_table<...>;      (or poggers::data_structs::tcf)
// switches to this library by including this header instead: the namespace
// alias makes every poggers::{tables,representations,insert_schemes,
// probing_schemes,hashers,sizing,data_structs,allocators} name resolve to the
// B200-native implementation with the same template parameters.
#pragma once
#include "poggers_b200/tables.cuh"
#include "poggers_b200/allocators.cuh"

namespace poggers = poggers_b200;
