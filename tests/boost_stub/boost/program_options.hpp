// Test-only stand-in for <boost/program_options.hpp>.
//
// The reference's command-line drivers (cppcode/aspl_cuda.cpp, piece2aspl.cpp,
// box2aspl.cpp, main.cpp, annealing.cpp) parse their options with Boost, which
// this image does not have.  To build those drivers from the reference sources,
// unchanged, against the engine's calculator shim, this header provides the
// part of Boost.Program_options' documented interface that they use, written
// from that interface's documentation (not from Boost's sources):
//   options_description(caption), add_options()(name[,value],help)...,
//   value<T>() -> typed_value<T>* with ->default_value(v),
//   variables_map with count(name) and [name].as<T>(),
//   store(parse_command_line(argc, argv, desc), vm), notify(vm),
//   error / error_with_option_name exceptions, and operator<< for the help text.
// Option names are "long,s" (long name, optional one-letter short name).  Accepted
// forms: --long value, --long=value, -s value, -svalue; a flag is an option without
// a value semantic.  Values convert with operator>> and must be consumed entirely.
#pragma once

#include <any>
#include <cassert>   // Boost's headers bring in assert(); annealing.cpp relies on it
#include <cstdlib>
#include <map>
#include <memory>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace boost {
namespace program_options {

class error : public std::logic_error {
public:
    explicit error(const std::string &what) : std::logic_error(what) {}
};

class error_with_option_name : public error {
public:
    error_with_option_name(const std::string &msg, const std::string &option)
        : error(msg + " (option '" + option + "')"), option_(option) {}
    const std::string &get_option_name() const { return option_; }

private:
    std::string option_;
};

// What an option's argument is: its type (conversion from text) and default.
class value_semantic {
public:
    virtual ~value_semantic() = default;
    virtual std::any parse(const std::string &text, const std::string &option) const = 0;
    virtual bool has_default() const = 0;
    virtual std::any default_any() const = 0;
    virtual std::string default_text() const = 0;
};

template <class T>
class typed_value : public value_semantic {
public:
    typed_value *default_value(const T &v) {
        def_ = v;
        has_def_ = true;
        std::ostringstream os;
        os << v;
        def_text_ = os.str();
        return this;
    }
    std::any parse(const std::string &text, const std::string &option) const override {
        if constexpr (std::is_same_v<T, std::string>) {
            return std::any(text);
        } else {
            std::istringstream is(text);
            T v{};
            is >> v;
            if (is.fail() || !(is >> std::ws).eof())
                throw error_with_option_name("the argument '" + text + "' is invalid", option);
            return std::any(v);
        }
    }
    bool has_default() const override { return has_def_; }
    std::any default_any() const override { return std::any(def_); }
    std::string default_text() const override { return def_text_; }

private:
    T def_{};
    bool has_def_ = false;
    std::string def_text_;
};

template <class T>
typed_value<T> *value() {
    return new typed_value<T>();
}

class option_description {
public:
    option_description(const std::string &names, const value_semantic *s, const std::string &help)
        : semantic_(s), help_(help) {
        const auto comma = names.find(',');
        long_ = names.substr(0, comma);
        if (comma != std::string::npos) short_ = names.substr(comma + 1);
    }
    const std::string &long_name() const { return long_; }
    const std::string &short_name() const { return short_; }
    const value_semantic *semantic() const { return semantic_.get(); }
    const std::string &description() const { return help_; }

private:
    std::string long_, short_;
    std::shared_ptr<const value_semantic> semantic_;
    std::string help_;
};

class options_description;

class options_description_easy_init {
public:
    explicit options_description_easy_init(options_description *owner) : owner_(owner) {}
    options_description_easy_init &operator()(const char *name, const char *help);
    options_description_easy_init &operator()(const char *name, const value_semantic *s, const char *help);

private:
    options_description *owner_;
};

class options_description {
public:
    explicit options_description(const std::string &caption = "") : caption_(caption) {}
    options_description_easy_init add_options() { return options_description_easy_init(this); }
    void add(const option_description &o) { options_.push_back(o); }
    const std::vector<option_description> &options() const { return options_; }
    const option_description *find(const std::string &name, bool is_short) const {
        for (const auto &o : options_)
            if ((is_short ? o.short_name() : o.long_name()) == name) return &o;
        return nullptr;
    }
    friend std::ostream &operator<<(std::ostream &os, const options_description &d) {
        os << d.caption_ << ":\n";
        for (const auto &o : d.options_) {
            os << "  ";
            if (!o.short_name().empty()) os << "-" << o.short_name() << " [ --" << o.long_name() << " ]";
            else os << "--" << o.long_name();
            if (o.semantic()) {
                os << " arg";
                if (o.semantic()->has_default()) os << " (=" << o.semantic()->default_text() << ")";
            }
            os << "  " << o.description() << "\n";
        }
        return os;
    }

private:
    std::string caption_;
    std::vector<option_description> options_;
};

inline options_description_easy_init &options_description_easy_init::operator()(const char *name,
                                                                                const char *help) {
    owner_->add(option_description(name, nullptr, help));
    return *this;
}
inline options_description_easy_init &options_description_easy_init::operator()(const char *name,
                                                                                const value_semantic *s,
                                                                                const char *help) {
    owner_->add(option_description(name, s, help));
    return *this;
}

class variable_value {
public:
    variable_value() = default;
    variable_value(std::any v, bool defaulted) : v_(std::move(v)), defaulted_(defaulted) {}
    template <class T>
    const T &as() const {
        return std::any_cast<const T &>(v_);
    }
    bool empty() const { return !v_.has_value(); }
    bool defaulted() const { return defaulted_; }

private:
    std::any v_;
    bool defaulted_ = false;
};

class variables_map : public std::map<std::string, variable_value> {};

// One parsed command line: (long option name, value) in order.
struct parsed_options {
    const options_description *description = nullptr;
    std::vector<std::pair<std::string, std::any>> values;
};

inline parsed_options parse_command_line(int argc, const char *const argv[], const options_description &d) {
    parsed_options p;
    p.description = &d;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        const option_description *o = nullptr;
        std::string text, shown = a;
        bool have_text = false;
        if (a.size() > 2 && a[0] == '-' && a[1] == '-') {
            const auto eq = a.find('=');
            const std::string name = a.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
            o = d.find(name, false);
            shown = name;
            if (eq != std::string::npos) { text = a.substr(eq + 1); have_text = true; }
        } else if (a.size() >= 2 && a[0] == '-') {
            o = d.find(a.substr(1, 1), true);
            shown = a.substr(0, 2);
            if (a.size() > 2) { text = a.substr(2); have_text = true; }
        } else {
            throw error_with_option_name("positional arguments are not accepted", a);
        }
        if (!o) throw error_with_option_name("unrecognised option", shown);
        if (!o->semantic()) {
            if (have_text) throw error_with_option_name("the option does not take an argument", shown);
            p.values.emplace_back(o->long_name(), std::any());
            continue;
        }
        if (!have_text) {
            if (i + 1 >= argc) throw error_with_option_name("the required argument is missing", shown);
            text = argv[++i];
        }
        p.values.emplace_back(o->long_name(), o->semantic()->parse(text, o->long_name()));
    }
    return p;
}

inline parsed_options parse_command_line(int argc, char *argv[], const options_description &d) {
    return parse_command_line(argc, const_cast<const char *const *>(argv), d);
}

// First value stored for a name wins (later store calls do not overwrite it);
// options with a default and no value on the command line get the default.
inline void store(const parsed_options &p, variables_map &vm) {
    for (const auto &kv : p.values) {
        auto it = vm.find(kv.first);
        if (it == vm.end() || it->second.defaulted()) vm[kv.first] = variable_value(kv.second, false);
    }
    if (p.description)
        for (const auto &o : p.description->options())
            if (o.semantic() && o.semantic()->has_default() && !vm.count(o.long_name()))
                vm[o.long_name()] = variable_value(o.semantic()->default_any(), true);
}

inline void notify(variables_map &) {}

}  // namespace program_options
}  // namespace boost
