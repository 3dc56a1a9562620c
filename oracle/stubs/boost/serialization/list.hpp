// Minimal stand-in for the two Boost.Serialization names the reference headers
// mention (`access` as a friend, `make_nvp` in never-instantiated templates).
// Serialization is never used on the hot path, so nothing here does any work.
#pragma once
namespace boost { namespace serialization {
class access {};
template <class T> inline T& make_nvp(const char*, T& t) { return t; }
}}
