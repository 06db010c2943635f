// gmsh 2.2 ASCII reader (reference src/geometry.cpp:307-957 reads the same
// sections: $PhysicalNames to map boundary names to conditions, $Nodes numbered
// 1..N in order, $Elements with the physical id as first tag).
#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <sstream>

#include "zb_internal.hpp"

namespace zb {

void MeshData::sync_view()
{
  view.coords = coords.data();
  view.ele2nodes = ele2nodes.data();
  view.face_nodes = face_nodes.empty() ? nullptr : face_nodes.data();
  view.face_bc = face_bc.empty() ? nullptr : face_bc.data();
}

static std::string lower(std::string s)
{
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  return s;
}

static int nodes_of_gmsh_type(int t)
{
  switch (t)
  {
    case 1: return 2;   // line2
    case 8: return 3;   // line3
    case 2: return 3;   // tri3
    case 9: return 6;   // tri6
    case 3: return 4;   // quad4
    case 10: return 9;  // quad9
    case 5: return 8;   // hex8
    case 12: return 27; // hex27
    case 4: return 4;   // tet4
    case 6: return 6;   // prism6
    default: return -1;
  }
}

void read_gmsh(const std::string &path, int ndims, const std::vector<std::string> &names,
               const std::vector<int> &bcs, MeshData &out)
{
  std::ifstream f(path);
  if (!f.is_open()) ZB_THROW(ZB_ERR_ARG, "could not open mesh file " + path);
  std::map<std::string, int> name_bc;
  for (size_t i = 0; i < names.size(); i++) name_bc[lower(names[i])] = bcs[i];

  std::map<int, int> phys_bc;  // gmsh physical id -> bc (or -1 for the volume)
  std::string line;
  bool have_nodes = false, have_eles = false;
  std::vector<std::vector<int64_t>> eles;
  int ele_type = -1;
  std::vector<std::vector<int64_t>> bfaces;
  std::vector<int> bface_bc;
  while (std::getline(f, line))
  {
    if (line.find("$PhysicalNames") != std::string::npos)
    {
      int n = 0;
      f >> n;
      std::getline(f, line);
      for (int i = 0; i < n; i++)
      {
        std::getline(f, line);
        std::stringstream ss(line);
        int dim = 0, id = 0;
        std::string nm;
        ss >> dim >> id >> nm;
        nm.erase(std::remove(nm.begin(), nm.end(), '"'), nm.end());
        std::string key = lower(nm);
        if (key == "fluid")
        {
          if (dim != ndims) ZB_THROW(ZB_ERR_MESH, "nDims in mesh file does not match the requested nDims");
          phys_bc[id] = -1;
          continue;
        }
        auto it = name_bc.find(key);
        if (it == name_bc.end()) ZB_THROW(ZB_ERR_MESH, "Unrecognized mesh boundary: \"" + key + "\"");
        phys_bc[id] = it->second;
      }
    }
    else if (line.find("$Nodes") != std::string::npos)
    {
      int64_t n = 0;
      f >> n;
      out.coords.assign((size_t)n * 3, 0.0);
      for (int64_t i = 0; i < n; i++)
      {
        int64_t id;
        double x, y, z;
        f >> id >> x >> y >> z;
        out.coords[i * 3 + 0] = x;
        out.coords[i * 3 + 1] = y;
        out.coords[i * 3 + 2] = (ndims == 3) ? z : 0.0;
      }
      out.view.n_nodes = n;
      have_nodes = true;
    }
    else if (line.find("$Elements") != std::string::npos)
    {
      int64_t n = 0;
      f >> n;
      std::getline(f, line);
      for (int64_t i = 0; i < n; i++)
      {
        std::getline(f, line);
        std::stringstream ss(line);
        int64_t id;
        int t, ntags;
        ss >> id >> t >> ntags;
        std::vector<int> tags(ntags);
        for (int k = 0; k < ntags; k++) ss >> tags[k];
        int nn = nodes_of_gmsh_type(t);
        if (nn < 0) ZB_THROW(ZB_ERR_MESH, "Unrecognized element type " + std::to_string(t));
        std::vector<int64_t> nd(nn);
        for (int k = 0; k < nn; k++)
        {
          ss >> nd[k];
          nd[k] -= 1;
        }
        bool is_face = (ndims == 2) ? (t == 1 || t == 8) : (t == 2 || t == 3 || t == 9 || t == 10);
        if (is_face)
        {
          int phys = ntags > 0 ? tags[0] : 0;
          auto it = phys_bc.find(phys);
          if (it == phys_bc.end()) ZB_THROW(ZB_ERR_MESH, "boundary face without a physical name");
          bfaces.push_back(nd);
          bface_bc.push_back(it->second);
        }
        else
        {
          if (ele_type >= 0 && ele_type != t) ZB_THROW(ZB_ERR_UNSUPPORTED, "mixed element types are not built");
          ele_type = t;
          eles.push_back(nd);
        }
      }
      have_eles = true;
    }
  }
  if (!have_nodes || !have_eles || eles.empty()) ZB_THROW(ZB_ERR_MESH, "mesh file missing $Nodes or $Elements");
  out.view.ndims = ndims;
  out.view.gmsh_type = ele_type;
  out.view.n_eles = (int64_t)eles.size();
  out.view.nodes_per_ele = nodes_of_gmsh_type(ele_type);
  out.ele2nodes.clear();
  out.ele2nodes.reserve(eles.size() * out.view.nodes_per_ele);
  for (auto &e : eles) out.ele2nodes.insert(out.ele2nodes.end(), e.begin(), e.end());
  int npf = 0;
  for (auto &b : bfaces) npf = std::max(npf, (int)b.size());
  out.view.nodes_per_face = npf;
  out.view.n_bnd_faces = (int64_t)bfaces.size();
  out.face_nodes.assign(bfaces.size() * (size_t)std::max(npf, 1), -1);
  for (size_t i = 0; i < bfaces.size(); i++)
    for (size_t k = 0; k < bfaces[i].size(); k++) out.face_nodes[i * npf + k] = bfaces[i][k];
  out.face_bc = bface_bc;
  out.sync_view();
}

}  // namespace zb
