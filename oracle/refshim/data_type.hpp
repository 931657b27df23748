// Test infrastructure: the column data types the reference's encoders switch on.  The reference
// takes this header from a data-manager submodule that its tree does not vendor; this stand-in
// declares the six types and the two helpers the encoders call, so that they compile here.  A
// serialised tree stores the type in each node header (tree/compression_node.cpp:84-90); the
// values are the library's own type codes (CHAR 0 .. DOUBLE 5), so that the reference's trees and
// the library's compare byte for byte.
#pragma once
#include <cstddef>
#include <ctime>
#include <string>

enum class DataType { d_char = 0, d_short = 1, d_int = 2, d_time = 3, d_float = 4, d_double = 5 };

inline size_t GetDataTypeSize(DataType type)
{
    switch (type) {
    case DataType::d_time: return sizeof(time_t);
    case DataType::d_char: return sizeof(char);
    case DataType::d_int: return sizeof(int);
    case DataType::d_float: return sizeof(float);
    case DataType::d_double: return sizeof(double);
    case DataType::d_short: return sizeof(short);
    }
    return 0;
}

inline std::string GetDataTypeString(DataType type)
{
    switch (type) {
    case DataType::d_time: return "time";
    case DataType::d_char: return "char";
    case DataType::d_int: return "int";
    case DataType::d_float: return "float";
    case DataType::d_double: return "double";
    case DataType::d_short: return "short";
    }
    return "unknown";
}
