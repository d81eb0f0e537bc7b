// No-op definitions of the reference's OutputFile members (OutputFile.h:105-131).
// The real ones (OutputFile.cpp) need the VTK library, which is not installed
// here; the harness dumps state itself instead of writing .vtu/.csv files.
// Test infrastructure only.
#include "OutputFile.h"

OutputFile::OutputFile(int outputIdx) : m_outputIdx(outputIdx) {}
OutputFile::~OutputFile() {}
void OutputFile::WriteVTK_Collective(SubDomain&) {}
void OutputFile::WriteVTK_LocalData(SubDomain&) {}
void OutputFile::WriteSurfaceAttribute(SubDomain&, int) {}
void OutputFile::processFlowData(const std::string&, const std::string&, double,
                                 const std::string&) {}
