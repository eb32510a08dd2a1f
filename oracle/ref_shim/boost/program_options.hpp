/*
Minimal stand-in for the part of boost::program_options used by the
reference's tests/mhd/reference.cpp (flags and one string option).
Written for this project; TEST INFRASTRUCTURE ONLY (oracle build recipe).
*/
#ifndef ORACLE_BOOST_PROGRAM_OPTIONS_STANDIN_HPP
#define ORACLE_BOOST_PROGRAM_OPTIONS_STANDIN_HPP

#include <cstdlib>
#include <iostream>
#include <map>
#include <set>
#include <string>
#include <type_traits>

namespace boost {
namespace program_options {

struct value_semantic {
	std::string* target = nullptr;
	value_semantic* default_value(const std::string&) { return this; }
};

template <class T> value_semantic* value(T* target)
{
	static_assert(std::is_same_v<T, std::string>, "only string options are supported");
	static value_semantic slots[16];
	static int used = 0;
	value_semantic* slot = &slots[used++ % 16];
	slot->target = target;
	return slot;
}

struct options_description;

struct option_adder {
	options_description* owner;
	option_adder& operator()(const char* name, const char* help);
	option_adder& operator()(const char* name, value_semantic* value, const char* help);
};

struct options_description {
	std::string caption;
	std::map<std::string, value_semantic*> valued;
	std::set<std::string> flags;
	explicit options_description(const std::string& c) : caption(c) {}
	option_adder add_options() { return option_adder{this}; }
};

inline option_adder& option_adder::operator()(const char* name, const char* /*help*/)
{
	owner->flags.insert(name);
	return *this;
}

inline option_adder& option_adder::operator()(
	const char* name, value_semantic* value, const char* /*help*/
) {
	owner->valued[name] = value;
	return *this;
}

struct parsed_options {
	const options_description* description = nullptr;
	std::map<std::string, std::string> values;
	std::set<std::string> seen;
};

inline parsed_options parse_command_line(int argc, char* argv[], const options_description& description)
{
	parsed_options parsed;
	parsed.description = &description;
	for (int i = 1; i < argc; i++) {
		std::string arg(argv[i]);
		if (arg.rfind("--", 0) != 0) {
			std::cerr << "unexpected argument " << arg << std::endl;
			std::exit(EXIT_FAILURE);
		}
		arg = arg.substr(2);
		std::string value;
		const auto eq = arg.find('=');
		if (eq != std::string::npos) {
			value = arg.substr(eq + 1);
			arg = arg.substr(0, eq);
		}
		if (description.valued.count(arg) > 0) {
			if (eq == std::string::npos) {
				if (i + 1 >= argc) {
					std::cerr << "missing value for --" << arg << std::endl;
					std::exit(EXIT_FAILURE);
				}
				value = argv[++i];
			}
			parsed.values[arg] = value;
		} else if (description.flags.count(arg) == 0) {
			std::cerr << "unknown option --" << arg << std::endl;
			std::exit(EXIT_FAILURE);
		}
		parsed.seen.insert(arg);
	}
	return parsed;
}

struct variables_map {
	std::set<std::string> seen;
	std::size_t count(const std::string& key) const { return seen.count(key); }
};

inline void store(const parsed_options& parsed, variables_map& map)
{
	map.seen.insert(parsed.seen.begin(), parsed.seen.end());
	for (const auto& item: parsed.values) {
		const auto slot = parsed.description->valued.find(item.first);
		if (slot != parsed.description->valued.end() and slot->second->target != nullptr) {
			*slot->second->target = item.second;
		}
	}
}

inline void notify(variables_map&) {}

inline std::ostream& operator<<(std::ostream& out, const options_description& description)
{
	return out << description.caption;
}

}} // namespaces

#endif
