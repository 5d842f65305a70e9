// Test-infrastructure shim: a minimal stand-in for the boost::format API that
// the reference's kriging sources use (construct from a pattern, feed values
// with operator%, read back with str() or operator<<).  Only the directive
// forms the reference writes are handled: %N% positional, %s / %d / %f
// sequential, and %% for a literal percent sign.
#ifndef ORACLE_SHIM_BOOST_FORMAT_HPP
#define ORACLE_SHIM_BOOST_FORMAT_HPP
#include <string>
#include <sstream>
#include <vector>
#include <ostream>
#include <cctype>

namespace boost {
class format {
    std::string pattern_;
    std::vector<std::string> args_;
public:
    explicit format(const std::string &p) : pattern_(p) {}
    explicit format(const char *p) : pattern_(p ? p : "") {}
    template <typename T> format &operator%(const T &v) {
        std::ostringstream os;
        os << v;
        args_.push_back(os.str());
        return *this;
    }
    std::string str() const {
        std::string out;
        size_t seq = 0;
        for (size_t i = 0; i < pattern_.size(); ++i) {
            char c = pattern_[i];
            if (c != '%' || i + 1 >= pattern_.size()) { out += c; continue; }
            char n = pattern_[i + 1];
            if (n == '%') { out += '%'; ++i; continue; }
            if (std::isdigit((unsigned char)n)) {
                size_t j = i + 1, num = 0;
                while (j < pattern_.size() && std::isdigit((unsigned char)pattern_[j]))
                    num = num * 10 + (pattern_[j++] - '0');
                if (j < pattern_.size() && pattern_[j] == '%' && num >= 1) {
                    if (num <= args_.size()) out += args_[num - 1];
                    i = j;
                    continue;
                }
            }
            if (std::isalpha((unsigned char)n)) {
                if (seq < args_.size()) out += args_[seq];
                ++seq;
                ++i;
                continue;
            }
            out += c;
        }
        return out;
    }
};
inline std::ostream &operator<<(std::ostream &os, const format &f) { return os << f.str(); }
inline std::string str(const format &f) { return f.str(); }
}  // namespace boost
#endif
