/*
 * olive_b200 source-compatible header layer: the reference's CommandLine
 * (commandLine.h:42-101): getArgument(i) is argv[i+1]; options are
 * "-name value" pairs.
 */
#ifndef OLIVE_COMMAND_LINE_H
#define OLIVE_COMMAND_LINE_H

#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

class CommandLine {
    int argc_;
    char **argv_;
    std::string usage_;

    const char *value(const std::string &opt) const {
        for (int i = 1; i < argc_ - 1; i++)
            if (opt == argv_[i]) return argv_[i + 1];
        return nullptr;
    }

public:
    CommandLine(int c, char **v, std::string s) : argc_(c), argv_(v), usage_(s) {}

    void badArgument() {
        std::cout << "usage: " << argv_[0] << " " << usage_ << std::endl;
        abort();
    }
    char *getArgument(int i) {
        if (argc_ < i + 2) badArgument();
        return argv_[i + 1];
    }
    bool getOption(std::string opt) {
        for (int i = 1; i < argc_; i++)
            if (opt == argv_[i]) return true;
        return false;
    }
    int getOptionIntValue(std::string opt, int dflt) {
        const char *v = value(opt);
        return v ? atoi(v) : dflt;
    }
    long getOptionLongValue(std::string opt, long dflt) {
        const char *v = value(opt);
        return v ? atol(v) : dflt;
    }
    double getOptionDoubleValue(std::string opt, double dflt) {
        const char *v = value(opt);
        if (!v) return dflt;
        double x;
        if (sscanf(v, "%lf", &x) != 1) badArgument();
        return x;
    }
};

#endif  // OLIVE_COMMAND_LINE_H
