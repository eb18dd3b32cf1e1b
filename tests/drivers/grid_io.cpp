// Reference-style use of DistUniformGrid's ingest and output through
// include/psp/psp.hpp (the calls the reference's examples make on their
// velocity models: SequentialLoad, InterpolateTo, WritePlane, WriteVolume).
//
//   grid_io write <dir>   WritePlane(XY, 1) and WriteVolume of a 6x5x4 grid
//   grid_io load <dir>    SequentialLoad of a ZYX file, InterpolateTo(11, 9, 7),
//                         the resampled buffer dumped to <dir>/resampled.bin
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>

#include "psp/psp.hpp"

static double Value(int x, int y, int z) { return 1.0 + 0.25 * x - 0.5 * y + 0.125 * x * z + 0.01 * y * y; }

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: grid_io write|load <dir>\n";
        return 2;
    }
    const std::string mode = argv[1], dir = argv[2];
    try {
        if (mode == "write") {
            psp::DistUniformGrid<double> g(6, 5, 4);
            for (int z = 0; z < 4; ++z)
                for (int y = 0; y < 5; ++y)
                    for (int x = 0; x < 6; ++x) g.Buffer()[g.LocalIndex(x, y, z)] = Value(x, y, z);
            g.WritePlane(psp::XY, 1, dir + "/plane");
            g.WriteVolume(dir + "/volume");
            return 0;
        }
        // a ZYX-ordered file: z fastest, then y, then x
        {
            std::ofstream f(dir + "/model_zyx.bin", std::ios::binary);
            for (int x = 0; x < 6; ++x)
                for (int y = 0; y < 5; ++y)
                    for (int z = 0; z < 4; ++z) {
                        const double v = Value(x, y, z);
                        f.write(reinterpret_cast<const char*>(&v), sizeof v);
                    }
        }
        psp::DistUniformGrid<double> g(6, 5, 4, 0, 1, psp::ZYX);
        g.SequentialLoad(dir + "/model_zyx.bin");
        g.InterpolateTo(11, 9, 7);
        std::ofstream out(dir + "/resampled.bin", std::ios::binary);
        out.write(reinterpret_cast<const char*>(g.LockedBuffer()), sizeof(double) * 11 * 9 * 7);
        std::cout << "resampled " << g.XSize() << " " << g.YSize() << " " << g.ZSize() << "\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
}
