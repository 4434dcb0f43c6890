// pf_fortfmt.h -- Fortran edit descriptors the reference's programs print
// and write with (host side of the main programs on the C-ABI).
#pragma once
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <string>

// Fortran E editing: Ew.d (0.ddddE+ee), right-justified in w
inline std::string fort_e(double x, int w, int d)
{
    char buf[64];
    if (x == 0.0) {
        std::snprintf(buf, sizeof buf, "0.%0*dE+00", d, 0);
    } else {
        char m[64];
        std::snprintf(m, sizeof m, "%.*E", d - 1, x);   // s.dddE+xx
        std::string ms(m);
        const size_t epos = ms.find('E');
        int ex = std::atoi(ms.c_str() + epos + 1) + 1;
        std::string digits;
        for (size_t q = 0; q < epos; ++q)
            if (std::isdigit((unsigned char)ms[q])) digits += ms[q];
        const char* sg = x < 0 ? "-" : "";
        if (std::abs(ex) <= 99)
            std::snprintf(buf, sizeof buf, "%s0.%sE%c%02d", sg, digits.c_str(), ex < 0 ? '-' : '+', std::abs(ex));
        else
            std::snprintf(buf, sizeof buf, "%s0.%s%c%03d", sg, digits.c_str(), ex < 0 ? '-' : '+', std::abs(ex));
    }
    std::string r(buf);
    if ((int)r.size() < w) r = std::string(w - r.size(), ' ') + r;
    return r;
}

// ES15.7E3 (saida.f90:54)
inline std::string fort_es15_7e3(double x)
{
    char m[64];
    std::snprintf(m, sizeof m, "%.7E", x);
    std::string ms(m);
    const size_t epos = ms.find('E');
    const int ex = std::atoi(ms.c_str() + epos + 1);
    char buf[64];
    std::snprintf(buf, sizeof buf, "%sE%c%03d", ms.substr(0, epos).c_str(), ex < 0 ? '-' : '+', std::abs(ex));
    std::string r(buf);
    if (r.size() < 15) r = std::string(15 - r.size(), ' ') + r;
    return r;
}

// Fortran ES editing: ESw.d (d.dddE+ee), right-justified in w
inline std::string fort_es(double x, int w, int d)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*E", d, x);
    std::string r(buf);
    if ((int)r.size() < w) r = std::string(w - r.size(), ' ') + r;
    return r;
}
