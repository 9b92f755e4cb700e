// Opm::ParameterGroup stand-in: the configuration object generated
// simulators build in main() (compiler/PrintCPUBackendASTVisitor.cpp:867-871
// in sintefmath/equelle emits `Opm::ParameterGroup param(argc, argv, false)`).
//
// Accepts `key=value` arguments and `*.param` files holding one `key=value`
// per line ('#' starts a comment), later settings overriding earlier ones,
// which is how the reference's tests and case kits configure runs
// (backends/cuda/CMakeLists.txt:88-93 passes a .param file as argv[1]).
#pragma once

#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace Opm {

class ParameterGroup {
public:
    ParameterGroup() = default;

    ParameterGroup(int argc, char** argv, bool verify_syntax = true)
    {
        (void)verify_syntax;
        for (int i = 1; i < argc; ++i) {
            const std::string arg = argv[i];
            const auto eq = arg.find('=');
            if (eq != std::string::npos) {
                insert(arg.substr(0, eq), arg.substr(eq + 1));
            } else if (arg.size() > 6 && arg.compare(arg.size() - 6, 6, ".param") == 0) {
                readParamFile(arg);
            } else {
                throw std::runtime_error("ParameterGroup: cannot interpret argument '" + arg + "'");
            }
        }
    }

    bool has(const std::string& key) const { return values_.count(key) > 0; }

    template <class T>
    T get(const std::string& key) const
    {
        auto it = values_.find(key);
        if (it == values_.end()) {
            throw std::runtime_error("ParameterGroup: missing parameter '" + key + "'");
        }
        return convert<T>(key, it->second);
    }

    template <class T>
    T getDefault(const std::string& key, const T& default_value) const
    {
        auto it = values_.find(key);
        if (it == values_.end()) {
            return default_value;
        }
        return convert<T>(key, it->second);
    }

    std::string getDefault(const std::string& key, const char* default_value) const
    {
        return getDefault<std::string>(key, std::string(default_value));
    }

    void insert(const std::string& key, const std::string& value)
    {
        if (!values_.count(key)) {
            order_.push_back(key);
        }
        values_[key] = value;
    }

    void readParamFile(const std::string& filename)
    {
        std::ifstream is(filename.c_str());
        if (!is) {
            throw std::runtime_error("ParameterGroup: could not open parameter file " + filename);
        }
        std::string line;
        while (std::getline(is, line)) {
            const auto hash = line.find('#');
            if (hash != std::string::npos) {
                line = line.substr(0, hash);
            }
            const auto eq = line.find('=');
            if (eq == std::string::npos) {
                continue;
            }
            insert(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
        }
    }

    // All settings in insertion order (the runtime forwards them over the C ABI).
    std::vector<std::pair<std::string, std::string>> items() const
    {
        std::vector<std::pair<std::string, std::string>> out;
        for (const auto& k : order_) {
            out.emplace_back(k, values_.at(k));
        }
        return out;
    }

private:
    static std::string trim(const std::string& s)
    {
        const auto b = s.find_first_not_of(" \t\r\n");
        if (b == std::string::npos) {
            return std::string();
        }
        const auto e = s.find_last_not_of(" \t\r\n");
        return s.substr(b, e - b + 1);
    }

    template <class T>
    static T convert(const std::string& key, const std::string& v)
    {
        std::istringstream is(v);
        T out{};
        is >> out;
        if (is.fail()) {
            throw std::runtime_error("ParameterGroup: cannot convert '" + v + "' for parameter '" + key + "'");
        }
        return out;
    }

    std::map<std::string, std::string> values_;
    std::vector<std::string> order_;
};

template <>
inline std::string ParameterGroup::convert<std::string>(const std::string&, const std::string& v)
{
    return v;
}

template <>
inline bool ParameterGroup::convert<bool>(const std::string& key, const std::string& v)
{
    if (v == "true" || v == "1" || v == "yes") {
        return true;
    }
    if (v == "false" || v == "0" || v == "no") {
        return false;
    }
    throw std::runtime_error("ParameterGroup: cannot convert '" + v + "' to bool for parameter '" + key + "'");
}

}  // namespace Opm
