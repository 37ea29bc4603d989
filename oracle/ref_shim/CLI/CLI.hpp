// Minimal stand-in for the CLI11 header that the reference's options header
// includes.  It exists only so the reference compiles into oracle/_ref for
// parity checks; command-line parsing through it always reports a parse error.
#pragma once
#include <exception>
#include <string>

namespace CLI {
struct Validator {};
static const Validator ExistingPath{};
static const Validator NonNegativeNumber{};
static const Validator PositiveNumber{};
inline Validator Range(double, double) { return Validator{}; }

struct Option {
    Option *required() { return this; }
    Option *check(const Validator &) { return this; }
};

struct ParseError : std::exception {
    const char *what() const noexcept override { return "command line parsing is not available"; }
};

struct App {
    std::string description;
    Option option;
    explicit App(std::string d) : description(std::move(d)) {}
    template <class T>
    Option *add_option(const std::string &, T &, const std::string & = "") { return &option; }
    Option *add_flag(const std::string &, bool &, const std::string & = "") { return &option; }
    void parse(int, char **) { throw ParseError(); }
    int exit(const ParseError &) { return 1; }
};
}  // namespace CLI
