// json.hpp -- TEST INFRASTRUCTURE ONLY: include/MC.hpp names nlohmann::json
// (an alias it never uses on the compiled path); this empty type stands in for
// the absent nlohmann_json library so src/MC.cpp compiles into oracle/_ref/.
#pragma once
namespace nlohmann {
struct json {};
}  // namespace nlohmann
