// Command-line flags of the demo programs: --key=value or --key value, bare
// --flag for booleans, --help. Unknown keys are errors.
#pragma once

#include <cstdlib>
#include <iostream>
#include <map>
#include <string>

namespace gs_native_demo {

class Args {
public:
    // spec: key -> default value ("" = required, "false" = boolean flag).
    Args(int argc, char** argv, std::map<std::string, std::string> spec) : values_(std::move(spec)) {
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a == "-h" || a == "--help" || a == "-?") {
                help_ = true;
                continue;
            }
            if (a.rfind("--", 0) != 0) {
                error_ = "unexpected argument " + a;
                continue;
            }
            a = a.substr(2);
            std::string value;
            const size_t eq = a.find('=');
            const std::string key = eq == std::string::npos ? a : a.substr(0, eq);
            auto it = values_.find(key);
            if (it == values_.end()) {
                error_ = "unknown flag --" + key;
                continue;
            }
            if (eq != std::string::npos) {
                value = a.substr(eq + 1);
            } else if (it->second == "false") {
                value = "true";
            } else if (i + 1 < argc) {
                value = argv[++i];
            } else {
                error_ = "missing value for --" + key;
                continue;
            }
            it->second = value;
        }
        for (const auto& kv : values_)
            if (kv.second.empty() && error_.empty()) error_ = "missing --" + kv.first;
    }
    bool help() const { return help_; }
    const std::string& error() const { return error_; }
    std::string str(const std::string& key) const { return values_.at(key); }
    int integer(const std::string& key) const { return std::atoi(values_.at(key).c_str()); }
    bool flag(const std::string& key) const { return values_.at(key) == "true"; }
    void usage(const char* about) const {
        std::cout << about << "\n";
        for (const auto& kv : values_)
            std::cout << "  --" << kv.first << (kv.second.empty() ? " (required)" : " [" + kv.second + "]") << "\n";
    }

private:
    std::map<std::string, std::string> values_;
    std::string error_;
    bool help_ = false;
};

}  // namespace gs_native_demo
