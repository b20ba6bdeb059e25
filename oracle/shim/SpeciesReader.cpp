// Replacement for the reference's Xerces-based src/SpeciesReader.cpp, used
// only when compiling the reference sources as the CPU oracle (oracle/_ref).
// Test infrastructure, not product.
//
// Reads the plain-text species format written by oracle/inputs.py (one
// keyword per line, arrays as a count followed by whitespace-separated
// values) and fills a Species through its `friend class SpeciesReader`
// access (src/Species.h:160), setting the same fields the SLPP branch of
// src/SpeciesHandler.cpp:120-248 sets from <species> XML.
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "Species.h"
#include "SpeciesReader.h"

using namespace std;

SpeciesReader::SpeciesReader(void) {}

void SpeciesReader::uri_to_species(const string uri, Species& sp)
{
  ifstream is(uri.c_str());
  if ( !is ) throw runtime_error("SpeciesReader: cannot open " + uri);
  string key;
  sp.type_ = Species::SLPP;
  sp.uri_ = uri;
  sp.description_ = "synthetic SLPP species";
  sp.nlcc_.clear();
  vector<vector<vector<double> > > d;
  while ( is >> key )
  {
    if ( key == "symbol" ) is >> sp.symbol_;
    else if ( key == "atomic_number" ) is >> sp.atomic_number_;
    else if ( key == "mass" ) is >> sp.mass_;
    else if ( key == "valence_charge" ) is >> sp.zval_;
    else if ( key == "lmax" ) is >> sp.lmax_;
    else if ( key == "mesh_spacing" ) is >> sp.deltar_;
    else if ( key == "local_potential" )
    {
      int n; is >> n;
      sp.vlocal_.resize(n);
      for ( int i = 0; i < n; i++ ) is >> sp.vlocal_[i];
    }
    else if ( key == "projector" )
    {
      int l, i, n; is >> l >> i >> n;
      if ( l >= (int) sp.proj_.size() ) sp.proj_.resize(l+1);
      if ( i >= (int) sp.proj_[l].size() ) sp.proj_[l].resize(i+1);
      sp.proj_[l][i].resize(n);
      for ( int k = 0; k < n; k++ ) is >> sp.proj_[l][i][k];
    }
    else if ( key == "d_ij" )
    {
      int l, i, j; double v; is >> l >> i >> j >> v;
      if ( l >= (int) d.size() ) d.resize(l+1);
      if ( i >= (int) d[l].size() ) d[l].resize(i+1);
      if ( j >= (int) d[l][i].size() ) d[l][i].resize(j+1, 0.0);
      d[l][i][j] = v;
    }
    else if ( key == "end" ) break;
    else throw runtime_error("SpeciesReader: unknown key " + key);
  }
  // a d_ij block exists for every l that has projectors (the SLPP check in
  // src/Species.cpp:534-565 requires proj_.size() == d_.size())
  if ( !d.empty() )
  {
    d.resize(sp.proj_.size());
    sp.d_ = d;
  }
}

void SpeciesReader::uri_to_string(const string uri, const string name,
  string& xmlstr)
{
  ifstream is(uri.c_str());
  ostringstream os; os << is.rdbuf();
  xmlstr = os.str();
}

void SpeciesReader::string_to_species(const string, Species&)
{
  throw runtime_error("SpeciesReader::string_to_species unsupported");
}
