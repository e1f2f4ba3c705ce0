// Stand-ins for the PDB-writer symbols defined in the reference's
// fileio/pdb.cpp, which the oracle build leaves out (that file does not
// compile with a current g++).  The oracle never writes PDB files; reaching
// any of these is a usage error and throws.
#include "global.h"
#include "fileio/pdb.h"
#include <stdexcept>

namespace IO {
static void no_pdb() { throw std::runtime_error("PDB output is not built into the test oracle"); }
PDBAtomLine::PDBAtomLine() {}
PDB_RawWriter::PDB_RawWriter() {}
void PDB_RawWriter::rawRemarks() const { no_pdb(); }
int PDB_RawWriter::rawWrite(const std::vector<PDBAtomLine> &, char, int) const { no_pdb(); return 0; }
PDB_Writer::PDB_Writer(const std::string &, bool) { no_pdb(); }
PDB_Writer::PDB_Writer(std::ostream &, bool) { no_pdb(); }
PDB_Writer::PDB_Writer(bool) { no_pdb(); }
void PDB_Writer::write(const MoleculeBase &) { no_pdb(); }
void PDB_Writer::write(const System &) { no_pdb(); }
}  // namespace IO
