// LSHKIT matrix I/O of kgraph-b200's kgraph-data.h (Matrix::load_lshkit /
// save_lshkit, the reference's kgraph-data.h:193-218 format): reads argv[1]
// as float32 and writes it back to argv[2]; reads argv[3] as uint32 and
// writes it back to argv[4].  Prints the shapes.  Host code only.
#include <kgraph.h>
#include <kgraph-data.h>
#include <cstdio>

int main(int argc, char **argv) {
    if (argc < 5) return 2;
    kgraph::Matrix<float> f;
    f.load_lshkit(argv[1]);
    f.save_lshkit(argv[2]);
    kgraph::Matrix<unsigned> u;
    u.load_lshkit(argv[3]);
    u.save_lshkit(argv[4]);
    bool rejects = false;
    try {
        kgraph::Matrix<double> wrong;   // element size 8 against a float32 file
        wrong.load_lshkit(argv[1]);
    } catch (kgraph::io_error const &) { rejects = true; }
    std::printf("f=%ux%u u=%ux%u rejects_wrong_size=%d\n", f.size(), f.dim(), u.size(), u.dim(), (int)rejects);
    return 0;
}
