#pragma once
// Clean-room stand-in for `cmd_line_parser::parser` (test infrastructure
// only; the reference's external/cmd_line_parser submodule is absent).  It
// supports what src/main.cpp:13-74 calls: add(name, help, shorthand,
// required, is_boolean), parse(), parsed(name), get<T>(name).

#include <cstdint>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace cmd_line_parser {

struct parser {
    parser(int argc, char** argv) : m_args(argv + 1, argv + argc), m_prog(argc ? argv[0] : "") {}

    void add(std::string const& name, std::string const& help, std::string const& shorthand,
             bool required, bool is_boolean = false) {
        m_opts.push_back({name, help, shorthand, required, is_boolean});
    }

    bool parse() {
        for (size_t i = 0; i < m_args.size(); ++i) {
            opt const* o = find_(m_args[i]);
            if (!o) {
                std::cerr << "unknown option " << m_args[i] << "\n";
                usage_();
                return false;
            }
            if (o->is_boolean) {
                m_values[o->name] = "true";
            } else {
                if (i + 1 >= m_args.size()) {
                    std::cerr << "missing value for " << m_args[i] << "\n";
                    return false;
                }
                m_values[o->name] = m_args[++i];
            }
        }
        for (auto const& o : m_opts) {
            if (o.required && !m_values.count(o.name)) {
                std::cerr << "missing required option " << o.shorthand << "\n";
                usage_();
                return false;
            }
        }
        return true;
    }

    bool parsed(std::string const& name) const { return m_values.count(name) != 0; }

    template <typename T>
    T get(std::string const& name) const {
        auto it = m_values.find(name);
        if (it == m_values.end()) return T();
        if constexpr (std::is_same<T, bool>::value) {
            return it->second == "true" || it->second == "1";
        } else if constexpr (std::is_same<T, std::string>::value) {
            return it->second;
        } else {
            std::istringstream is(it->second);
            T v{};
            is >> v;
            return v;
        }
    }

private:
    struct opt {
        std::string name, help, shorthand;
        bool required, is_boolean;
    };
    opt const* find_(std::string const& s) const {
        for (auto const& o : m_opts)
            if (o.shorthand == s) return &o;
        return nullptr;
    }
    void usage_() const {
        std::cerr << "usage: " << m_prog << "\n";
        for (auto const& o : m_opts)
            std::cerr << "  " << o.shorthand << "  " << o.name << (o.required ? " (required)" : "")
                      << "\n";
    }
    std::vector<std::string> m_args;
    std::string m_prog;
    std::vector<opt> m_opts;
    std::map<std::string, std::string> m_values;
};

}  // namespace cmd_line_parser
