// kpax_io.cpp — host-side environment input: the reference's obstacle CSV files.
//
// readObstaclesFromCSV (src/helper/helper.cu:13-39) reads a file line by line and takes floats off
// each line by stream extraction, skipping one comma after each value; the first token that does
// not extract as a float ends its line.  Files written for the reference (include/config/obstacles/*)
// and malformed ones (headers, empty fields, spaces before commas, a trailing partial row) therefore
// read here exactly as there: the same token rule, through the same standard-library extraction.
#include <stdint.h>

#include <fstream>
#include <new>
#include <sstream>
#include <string>

#include "kpax_params.h"

using namespace kpax;

extern "C" {

kpax_status kpax_read_obstacles_csv(const char* filename, float* h_values, uint64_t capacity, uint64_t* n_values)
{
    if(!filename || !n_values) return set_error("kpax_read_obstacles_csv: null argument"), KPAX_EINVAL;
    *n_values = 0;
    try {
        std::ifstream file(filename);
        if(!file.is_open()) return set_error("kpax_read_obstacles_csv: cannot open %s", filename), KPAX_EINVAL;
        uint64_t n = 0;
        std::string line;
        while(std::getline(file, line)) {
            std::istringstream fields(line);
            for(float v; fields >> v; ++n) {
                if(h_values && n < capacity) h_values[n] = v;
                if(fields.peek() == ',') fields.get();
            }
        }
        *n_values = n;
        return KPAX_OK;
    } catch(const std::bad_alloc&) {
        return set_error("kpax_read_obstacles_csv: out of host memory"), KPAX_ENOMEM;
    } catch(const std::exception& e) {
        return set_error("kpax_read_obstacles_csv: %s", e.what()), KPAX_EINVAL;
    }
}

}  // extern "C"
