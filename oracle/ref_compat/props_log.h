// Compatibility measure for building the reference's render loop with GCC —
// TEST INFRASTRUCTURE ONLY.  Force-included (g++ -include) into the
// translation units of oracle/Makefile's refloop target.
//
// The reference's `std::ostream& operator<<(std::ostream&, const Props&)`
// (sys/props.h:170-181) ends without returning its stream.  Flowing off the
// end of a value-returning function is undefined behaviour; GCC 13 compiles
// it to a trap (-O0) or to code that runs into whatever follows (-O2), so the
// render loop dies at its first `Log() << props` (render_window.cpp's
// printFrameStats and onDestroy).  Log messages write into the
// std::ostringstream of LogMessage (sys/logging.h:31-47); this overload for
// that exact stream type is a better match than the reference's one for
// std::ostream, prints the same "name=value" pairs separated by spaces, and
// returns its stream.  No reference file is edited.
#pragma once

#include <sstream>

#include "sys/props.h"

namespace prt {

inline std::ostringstream& operator<<(std::ostringstream& osm, const Props& props)
{
    bool first = true;
    for (auto& entry : props)
    {
        if (!first) osm << " ";
        first = false;
        osm << entry.first << "=" << entry.second;
    }
    return osm;
}

} // namespace prt
