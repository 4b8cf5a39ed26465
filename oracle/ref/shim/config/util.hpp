// Oracle shim for DACTI's config/util.hpp (src/lib/config/util.hpp).
//
// The model headers only reach this file from their `dict()` members, which parse a TOML case
// file (e.g. model/euler.hpp:288-324). The oracle runner never parses TOML: it sets the model
// constants directly. This stub declares just enough of the toml++ surface for those members to
// compile; calling `get_entry` without a default raises, so a stray TOML read fails loudly.
#pragma once

#include <core/util.hpp>
#include <dacti.hpp>
#include <optional>
#include <stdexcept>
#include <string>

namespace toml {
	struct table;
	struct node {};

	template<typename N>
	struct node_view {
		node_view operator[](const char *) const { return {}; }
		explicit operator bool() const { return false; }
		table *as_table() const { return nullptr; }
	};

	struct table {
		node_view<node> operator[](const char *) const { return {}; }
		bool contains(const char *) const { return false; }
	};
}    // namespace toml

namespace dacti::config {
	template<typename T>
	T get_entry(const toml::table &, const std::string &path, std::optional<T> default_value = std::nullopt) {
		if (default_value) return *default_value;
		throw std::runtime_error("oracle runner does not parse case files (entry '" + path + "')");
	}
}    // namespace dacti::config
