// purgeJournal: compact a crash journal.
// Reference: purgeJournal.cpp (options :27-50, main :52-75) over
// Journal::loadMemo / purgeMemo (GatlasBenchmark.cpp:56-105): keeps the
// records of bad keys (no time: crashed while building or hung while
// running) and, unless -d, the run state and times of the good keys.
#include <unistd.h>

#include <cstdlib>
#include <iostream>
#include <string>

#include "host/bench.hpp"

using namespace gatlas::host;
using std::cerr;
using std::cout;
using std::endl;

int main(int argc, char **argv) {
    std::string journalFile;
    bool deleteTimes = false;
    int opt;
    while ((opt = getopt(argc, argv, "hdj:")) != -1) {
        switch (opt) {
            case 'h':
                cerr << "usage: " << argv[0] << " -j journalFile [-d] [-h]" << endl
                     << "\t-j journal file" << endl
                     << "\t-d delete benchmark time records for good kernels (default is to keep them)" << endl
                     << "\t-h help" << endl;
                exit(1);
            case 'j': journalFile = optarg; break;
            case 'd': deleteTimes = true; break;
        }
    }
    if (journalFile.empty()) {
        cerr << "error: journal file must be specified" << endl;
        exit(1);
    }
    Journal journal(journalFile);
    if (journal.loadMemo()) {
        const size_t good = journal.memoGood();
        const int bad = journal.purgeMemo(deleteTimes);
        cout << "journal file " << journalFile << " has " << bad << " bad keys, "
             << (deleteTimes ? "deleted " : "preserved ") << good << " good keys" << endl;
    } else {
        cerr << "error: could not load journal file " << journalFile << endl;
    }
    return 0;
}
