// Replacement for sparselizard's src/formulation/contribution.cpp (same
// header, contribution.h, unchanged).
//
// generate() no longer multiplies dense matrices on the host.  For every
// group of disjoint regions with the same element type and dof/tf orders it
// lowers the contribution into an slgpu_group:
//   - the Gauss points, weights and Lagrange geometry tables of the group,
//   - the form-function tables of every term, one copy per total orientation,
//   - one coefficient program (a DAG over J, invJ, detJ, constants,
//     per-element parameter values and field coefficients) for all terms,
//   - the harmonic folding of contribution.cpp:213-246 as per-term scales,
//   - the dof/tf addresses from dofmanager::getaddresses per harmonic block,
// and hands it to the engine: matrix groups are recorded in the rawmat's
// engine matrix (assembled in rawmat::process), right-hand-side groups are
// assembled immediately and added to the rawvec.
//
// The grouping, integration order, Gauss rule, orientation handling and
// harmonic rules follow the reference implementation step by step
// (src/formulation/contribution.cpp:20-308) because they define which
// entries exist and their values.  Anything the engine does not implement
// raises an error; nothing is computed on the host as a fallback.
#include "contribution.h"

#include "dofinterpolate.h"
#include "lagrangeformfunction.h"
#include "opharmonic.h"
#include "slgpu_adapter.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <tuple>
#include <sstream>
#include <typeinfo>

contribution::contribution(std::shared_ptr<dofmanager> dofmngr) { mydofmanager = dofmngr; }

void contribution::setdofs(std::vector<std::shared_ptr<operation>> dofs) { mydofs = dofs; }
void contribution::settfs(std::vector<std::shared_ptr<operation>> tfs) { mytfs = tfs; }
void contribution::setcoeffs(std::vector<std::shared_ptr<operation>> coeffs) { mycoeffs = coeffs; }
void contribution::setdoffield(std::shared_ptr<rawfield> input) { doffield = input; }
void contribution::settffield(std::shared_ptr<rawfield> input) { tffield = input; }
void contribution::setmeshdeformation(expression meshdeform) { mymeshdeformation = {meshdeform}; }
void contribution::setintegrationphysicalregion(int physreg) { integrationphysreg = physreg; }
void contribution::setdofphysicalregion(int physreg) { dofphysreg = physreg; }
void contribution::settfphysicalregion(int physreg) { tfphysreg = physreg; }
void contribution::setintegrationorderdelta(int integrorderdelta) { integrationorderdelta = integrorderdelta; }
void contribution::setnumfftcoeffs(int numcoeffs) { numfftcoeffs = numcoeffs; }
void contribution::setbarycenterevalflag(void) { isbarycentereval = true; }



namespace {

[[noreturn]] void unsupported(const std::string& what)
{
    logs log;
    log.msg() << "Error in the GPU assembly engine: " << what << " is not supported" << std::endl;
    log.error();
    throw std::runtime_error(what);
}

// Text printed by an operation's print() (used to read opjac/opinvjac indices,
// which the operation classes keep private).
std::string printed(const std::shared_ptr<operation>& op)
{
    std::stringstream ss;
    std::streambuf* old = std::cout.rdbuf(ss.rdbuf());
    op->print();
    std::cout.rdbuf(old);
    return ss.str();
}

// opharmonic (sl::moveharmonic, src/expression/operation/sl.cpp:555-601) keeps
// its harmonic maps private and has no getters.  An explicit instantiation
// may name private members (access is not checked there), which gives read
// access through these pointers-to-member.
template <class Tag, typename Tag::type M>
struct MemberAccess {
    friend typename Tag::type member(Tag) { return M; }
};
struct HarmOrig {
    typedef std::vector<int> opharmonic::*type;
    friend type member(HarmOrig);
};
struct HarmDest {
    typedef std::vector<int> opharmonic::*type;
    friend type member(HarmDest);
};
struct HarmFft {
    typedef int opharmonic::*type;
    friend type member(HarmFft);
};
template struct MemberAccess<HarmOrig, &opharmonic::myorigharms>;
template struct MemberAccess<HarmDest, &opharmonic::mydestharms>;
template struct MemberAccess<HarmFft, &opharmonic::mynumfftharms>;

// DOF addresses of one (dofmanager, field, order, element type, element list,
// region), kept across assemblies: the slices of a vector field's formulation
// ask for the same test-function and dof addresses many times (elasticity: 18
// requests, 6 distinct tables), and a repeated generate() asks for them again.
// The addresses depend on the dofmanager's numbering, which changes only when
// the mesh number changes or a field is added (dofmanager.cpp:4-33, ndofs
// changes then), and on the field's interpolation order on each disjoint
// region.  An entry therefore holds the dofmanager and field themselves (weak
// references: a destroyed object never matches a new one at the same address),
// its key holds the mesh number, ndofs, the element list's hash and the
// field's orders, and every hit is still checked against a fresh lookup of 64
// elements spread over the list.
struct AddressKey {
    const void* dm;
    const void* field;
    int order, elemtype, physreg, meshnumber;
    long long ndofs;
    size_t n;
    unsigned long long hash, orders;
    bool operator<(const AddressKey& o) const
    {
        return std::tie(dm, field, order, elemtype, physreg, meshnumber, ndofs, n, hash, orders) <
               std::tie(o.dm, o.field, o.order, o.elemtype, o.physreg, o.meshnumber, o.ndofs, o.n, o.hash, o.orders);
    }
};
struct AddressEntry {
    std::weak_ptr<dofmanager> dm;
    std::weak_ptr<rawfield> field;
    indexmat addresses;
};
std::map<AddressKey, AddressEntry> g_address_cache;
constexpr size_t kAddressEntries = 64;
constexpr int kAddressProbe = 64;

indexmat cached_addresses(const std::shared_ptr<dofmanager>& dm, const std::shared_ptr<rawfield>& f, int order, int elemtype,
                          std::vector<int>& elems, int physreg)
{
    unsigned long long h = 1469598103934665603ull;
    for (int e : elems) h = (h ^ (unsigned long long)(unsigned)e) * 1099511628211ull;
    unsigned long long orders = 1469598103934665603ull;
    for (int d : universe::getrawmesh()->getphysicalregions()->get(physreg)->getdisjointregions(-1))
        orders = (orders ^ ((unsigned long long)(unsigned)d << 8 | (unsigned)f->getinterpolationorder(d))) * 1099511628211ull;
    const AddressKey key{dm.get(), f.get(), order, elemtype, physreg, universe::getrawmesh()->getmeshnumber(), dm->countdofs(),
                         elems.size(), h, orders};
    auto it = g_address_cache.find(key);
    if (it != g_address_cache.end() && !elems.empty()) {
        bool same = it->second.dm.lock() == dm && it->second.field.lock() == f;
        if (same) {
            const long long n = (long long)elems.size(), np = std::min<long long>(n, kAddressProbe);
            std::vector<int> probe(np);
            std::vector<long long> col(np);
            for (long long i = 0; i < np; i++) {
                col[i] = np > 1 ? i * (n - 1) / (np - 1) : 0;
                probe[i] = elems[col[i]];
            }
            indexmat fresh = dm->getaddresses(f, order, elemtype, probe, physreg);
            indexmat c = it->second.addresses;
            const long long rows = c.countrows();
            same = fresh.countrows() == rows && c.countcolumns() == n;
            for (long long r = 0; same && r < rows; r++)
                for (long long i = 0; same && i < np; i++) same = fresh.getvalues()[r * np + i] == c.getvalues()[r * n + col[i]];
        }
        if (same)
            return it->second.addresses;
        g_address_cache.erase(it);
    }
    indexmat a = dm->getaddresses(f, order, elemtype, elems, physreg);
    if (g_address_cache.size() >= kAddressEntries)
        g_address_cache.clear();
    g_address_cache[key] = AddressEntry{dm, f, a};
    return a;
}

// Elements of a disjoint-region group in orientation groups (the lists that
// elementselector hands out, concatenated, with each element's variant and the
// variants' total orientations), kept per mesh and region list: they depend
// only on the mesh's elements, which a mesh number change (adaptation)
// renews.  Holds the rawmesh weakly, so that a new mesh at the address of a
// destroyed one never matches.
struct SelectorKey {
    const void* mesh;
    int meshnumber;
    bool orientdep;
    std::vector<int> disjregs;
    bool operator<(const SelectorKey& o) const
    {
        return std::tie(mesh, meshnumber, orientdep, disjregs) < std::tie(o.mesh, o.meshnumber, o.orientdep, o.disjregs);
    }
};
struct SelectorEntry {
    std::weak_ptr<rawmesh> mesh;
    std::vector<int> elems, variant, totalorients;
};
std::map<SelectorKey, SelectorEntry> g_selector_cache;
constexpr size_t kSelectorEntries = 16;

// Lowers coefficient operation trees of one disjoint-region group into an
// slgpu coefficient program.  Shared subtrees (same operation object) become
// one node.
class Lowering {
public:
    std::vector<slgpu_node> nodes;
    std::vector<double> consts;
    std::vector<std::vector<double>> elemdata;
    std::vector<std::vector<double>> fielddata;
    std::vector<int32_t> fieldrows;
    // Extra tables needed by field nodes: (name, table [norient][rows][ngp]).
    std::vector<std::vector<double>> fieldtables;
    std::vector<int32_t> fieldtablerows;

    Lowering(const std::vector<int>& disjregs, int elemtype, const std::vector<int>& elems, const std::vector<int>& orientvariant,
             const std::vector<int>& totalorientations, std::vector<double>& gpcoords)
        : disjregs_(disjregs), elemtype_(elemtype), elems_(elems), variant_(orientvariant), orients_(totalorientations), gp_(gpcoords)
    {
    }

    int lower(const std::shared_ptr<operation>& op)
    {
        auto it = memo_.find(op.get());
        if (it != memo_.end())
            return it->second;
        int n = lower_new(op);
        memo_[op.get()] = n;
        return n;
    }

    // Offsets of field tables within the group's table list are assigned by the caller.
    int field_table_base = 0;

private:
    const std::vector<int>& disjregs_;
    int elemtype_;
    const std::vector<int>& elems_;
    const std::vector<int>& variant_;
    const std::vector<int>& orients_;
    std::vector<double>& gp_;
    std::map<const operation*, int> memo_;
    std::map<double, int> constmemo_;

    int add(int op, int a = 0, int b = 0)
    {
        nodes.push_back(slgpu_node{op, a, b, 0});
        return (int)nodes.size() - 1;
    }

    int constant(double v)
    {
        auto it = constmemo_.find(v);
        int idx;
        if (it == constmemo_.end() || std::signbit(v) != std::signbit(it->first)) {
            idx = (int)consts.size();
            consts.push_back(v);
            constmemo_[v] = idx;
        } else
            idx = it->second;
        return add(SLGPU_OP_CONST, idx);
    }

    int chain(int op, const std::vector<std::shared_ptr<operation>>& args)
    {
        if (args.empty())
            unsupported("an empty sum/product in a coefficient");
        int acc = lower(args[0]);
        for (size_t i = 1; i < args.size(); i++) acc = add(op, acc, lower(args[i]));
        return acc;
    }

    int lower_new(const std::shared_ptr<operation>& op)
    {
        operation* p = op.get();
        if (op->isconstant())
            return constant(op->getvalue());
        if (op->issum())
            return chain(SLGPU_OP_ADD, op->getarguments());
        if (op->isproduct())
            return chain(SLGPU_OP_MUL, op->getarguments());
        if (dynamic_cast<opinvjac*>(p) != nullptr || dynamic_cast<opjac*>(p) != nullptr) {
            bool inv = dynamic_cast<opinvjac*>(p) != nullptr;
            std::string s = printed(op);
            if (s.size() < 2)
                unsupported("an unreadable Jacobian term");
            int r = s[s.size() - 2] - '0', c = s[s.size() - 1] - '0';
            if (r < 0 || r > 2 || c < 0 || c > 2)
                unsupported("a Jacobian term with indices '" + s + "'");
            return add(inv ? SLGPU_OP_INVJAC : SLGPU_OP_JAC, r, c);
        }
        if (dynamic_cast<opdetjac*>(p) != nullptr)
            return add(SLGPU_OP_DETJAC);
        if (dynamic_cast<opinversion*>(p) != nullptr)
            return add(SLGPU_OP_INV, lower(op->getarguments()[0]));
        if (dynamic_cast<oppower*>(p) != nullptr) {
            auto a = op->getarguments();
            int b = lower(a[0]);
            int e = lower(a[1]);
            return add(SLGPU_OP_POW, b, e);
        }
        if (op->isparameter())
            return parameter(op);
        if (op->isfield())
            return fieldvalue(op);
        if (auto* h = dynamic_cast<opharmonic*>(p))
            return moved_harmonic(*h);
        unsupported(std::string("the coefficient operation '") + typeid(*p).name() + "'");
    }

    // opharmonic (opharmonic.cpp:12-57): harmonic dest_i of the result sums
    // harmonic orig_i of the argument.  Coefficients here are constant in
    // time (harmonic 1 only), so with every destination harmonic 1 and an
    // argument of harmonic 1 the result is k times the argument, k the number
    // of pairs (1 -> 1): what setvalue / setconstraint produce for a field
    // that is not multiharmonic (sl::getharmonic(1, expr)).
    int moved_harmonic(opharmonic& h)
    {
        const std::vector<int>& orig = h.*member(HarmOrig());
        const std::vector<int>& dest = h.*member(HarmDest());
        if (h.*member(HarmFft()) >= 0)
            unsupported("FFT-based harmonic extraction in a coefficient");
        std::shared_ptr<operation> arg = h.getarguments()[0];
        if (!arg->isharmonicone(disjregs_))
            unsupported("a harmonic of a multiharmonic coefficient");
        int k = 0;
        for (size_t i = 0; i < orig.size(); i++) {
            if (dest[i] != 1)
                unsupported("a coefficient moved to a harmonic other than 1");
            k += orig[i] == 1 ? 1 : 0;
        }
        if (k == 0)
            return constant(0.0);
        const int a = lower(arg);
        return k == 1 ? a : add(SLGPU_OP_MUL, constant((double)k), a);
    }

    // opparameter: one expression per disjoint region (opparameter.cpp:4).
    int parameter(const std::shared_ptr<operation>& op)
    {
        std::shared_ptr<rawparameter> rp = op->getparameterpointer();
        int row = op->getselectedrow(), col = op->getselectedcol();
        std::vector<std::shared_ptr<operation>> perreg;
        bool allconst = true, allsame = true;
        for (int dr : disjregs_) {
            std::shared_ptr<operation> o = rp->get(dr, row, col);
            if (o == nullptr)
                unsupported("a parameter undefined on part of the integration region");
            perreg.push_back(o);
            allconst = allconst && o->isconstant();
            allsame = allsame && o.get() == perreg[0].get();
        }
        if (allsame)
            return lower(perreg[0]);
        if (!allconst)
            unsupported("a parameter with different non-constant expressions on the disjoint regions of one element group");
        std::map<int, double> value;
        for (size_t i = 0; i < disjregs_.size(); i++) value[disjregs_[i]] = perreg[i]->getvalue();
        elements* els = universe::getrawmesh()->getelements();
        std::vector<double> v(elems_.size());
        for (size_t e = 0; e < elems_.size(); e++) v[e] = value.at(els->getdisjointregion(elemtype_, elems_[e]));
        elemdata.push_back(std::move(v));
        return add(SLGPU_OP_ELEM, (int)elemdata.size() - 1);
    }

    // opfield without derivatives: coefficients x form functions
    // (rawfield::interpolate, src/field/rawfield.cpp:2632-2686).
    int fieldvalue(const std::shared_ptr<operation>& op)
    {
        std::shared_ptr<rawfield> f = op->getfieldpointer();
        if (op->getspacederivative() != 0 || op->getkietaphiderivative() != 0)
            unsupported("a derivative of a field inside a coefficient");
        if (op->gettimederivative() != 0)
            unsupported("a time derivative of a field inside a coefficient");
        std::string tn = f->gettypename();
        if (tn == "x" || tn == "y" || tn == "z")
            return add(SLGPU_OP_COORD, tn == "x" ? 0 : (tn == "y" ? 1 : 2));
        // The coefficients live in the harmonic-1 subfield (harmonic(1) of a
        // field without harmonics is the field itself, rawfield.cpp:1776-1778).
        std::vector<int> h = f->getharmonics();
        if (!(h.size() == 1 && h[0] == 1))
            unsupported("a multiharmonic field inside a coefficient");
        f = f->harmonic(1);
        int order = f->getinterpolationorder(disjregs_[0]);
        for (int dr : disjregs_)
            if (f->getinterpolationorder(dr) != order)
                unsupported("a coefficient field with different orders inside one element group");
        densemat coefs = f->getcoefficients(elemtype_, order, const_cast<std::vector<int>&>(elems_));
        int rows = coefs.countrows();
        fielddata.emplace_back(coefs.getvalues(), coefs.getvalues() + (size_t)rows * coefs.countcolumns());
        fieldrows.push_back(rows);
        hierarchicalformfunctioncontainer* val = universe::gethff(f->gettypename(), elemtype_, order, gp_);
        int ngp = (int)gp_.size() / 3;
        std::vector<double> tab((size_t)orients_.size() * rows * ngp);
        for (size_t o = 0; o < orients_.size(); o++) {
            densemat m = val->tomatrix(orients_[o], order, 0, op->getformfunctioncomponent());
            if (m.countrows() != rows || m.countcolumns() != ngp)
                unsupported("a coefficient field whose form functions do not match its coefficients");
            std::copy(m.getvalues(), m.getvalues() + (size_t)rows * ngp, tab.begin() + (size_t)o * rows * ngp);
        }
        fieldtables.push_back(std::move(tab));
        fieldtablerows.push_back(rows);
        return add(SLGPU_OP_FIELD, (int)fielddata.size() - 1, field_table_base + (int)fieldtables.size() - 1);
    }
};

struct TableKey {
    bool istf;
    int deriv, comp;
    bool operator<(const TableKey& o) const
    {
        return std::tie(istf, deriv, comp) < std::tie(o.istf, o.deriv, o.comp);
    }
};

}  // namespace

void contribution::generate(std::shared_ptr<rawvec> myvec, std::shared_ptr<rawmat> mymat)
{
    if (doffield != NULL && mydofs[0]->ison())
        unsupported("dof interpolation on another region (on())");
    if (numfftcoeffs > 0)
        unsupported("FFT-based multiharmonic coefficients");
    if (mymeshdeformation.size() > 0)
        unsupported("integration on a deformed mesh");
    if (universe::isaxisymmetric)
        unsupported("axisymmetry");
    if (doffield == NULL && universe::keeptrackofrhsassembly)
        unsupported("right-hand-side assembly tracking");

    slgpu_ctx* ctx = slgpu_adapter::context();
    const int prec = slgpu_adapter::precision();
    const int meshdim = universe::getrawmesh()->getmeshdimension();
    const long long ndofs = mydofmanager->countdofs();

    std::vector<int> tfharms = tffield->getharmonics();
    std::vector<int> dofharms = {1};
    if (doffield != NULL)
        dofharms = doffield->getharmonics();

    std::vector<bool> isnodeintfphysreg;
    if (tfphysreg != integrationphysreg)
        universe::getrawmesh()->getelements()->istypeindisjointregions(
            0, universe::getrawmesh()->getphysicalregions()->get(tfphysreg)->getdefinition(), isnodeintfphysreg, false);

    std::vector<int> selectedelemdisjregs = universe::getrawmesh()->getphysicalregions()->get(integrationphysreg)->getdisjointregions();
    std::vector<int> tfinterpolorders(selectedelemdisjregs.size());
    std::vector<int> dofinterpolorders(selectedelemdisjregs.size(), 0);
    for (size_t i = 0; i < selectedelemdisjregs.size(); i++) {
        tfinterpolorders[i] = tffield->getinterpolationorder(selectedelemdisjregs[i]);
        if (doffield != NULL)
            dofinterpolorders[i] = doffield->getinterpolationorder(selectedelemdisjregs[i]);
    }

    disjointregionselector mydisjregselector(selectedelemdisjregs, {tfinterpolorders, dofinterpolorders});
    for (int grp = 0; grp < mydisjregselector.countgroups(); grp++) {
        std::vector<int> mydisjregs = mydisjregselector.getgroup(grp);
        const int elemtype = universe::getrawmesh()->getdisjointregions()->getelementtypenumber(mydisjregs[0]);
        const int tforder = tffield->getinterpolationorder(mydisjregs[0]);
        const int doforder = doffield != NULL ? doffield->getinterpolationorder(mydisjregs[0]) : tforder;
        // Barycenter evaluation (contribution.cpp:77-78,175-176,199-200): order 0,
        // neither weights nor det J applied.  On point elements (the nodal
        // Dirichlet projection, rawfield.cpp:134-162) that is the plain point
        // value: one point of weight 1, identity Jacobian.
        const int integrationorder = isbarycentereval ? 0 : doforder + tforder + 2 + integrationorderdelta;
        if (integrationorder < 0) {
            logs log;
            log.msg() << "Error in 'contribution' object: trying to integrate at negative order " << integrationorder << std::endl;
            log.error();
        }
        element elemobj(elemtype);
        const int elemdim = elemobj.getelementdimension();
        if (isbarycentereval && elemdim != 0)
            unsupported("barycenter evaluation on elements other than points");

        gausspoints gps(elemtype, integrationorder);
        std::vector<double> gpcoords = gps.getcoordinates();
        std::vector<double> weights = gps.getweights();
        if (isbarycentereval)
            std::fill(weights.begin(), weights.end(), 1.0);
        const int ngp = (int)weights.size();

        std::shared_ptr<hierarchicalformfunction> tfff = selector::select(elemtype, tffield->gettypename());
        hierarchicalformfunctioncontainer tfval = *(universe::gethff(tffield->gettypename(), elemtype, tforder, gpcoords));
        std::shared_ptr<hierarchicalformfunction> dofff;
        hierarchicalformfunctioncontainer dofval;
        if (doffield != NULL) {
            dofff = selector::select(elemtype, doffield->gettypename());
            dofval = *(universe::gethff(doffield->gettypename(), elemtype, doforder, gpcoords));
        }

        bool isorientationdependent = tfff->isorientationdependent(tforder);
        if (doffield != NULL)
            isorientationdependent = isorientationdependent || dofff->isorientationdependent(doforder);
        std::vector<std::shared_ptr<operation>> coefs(mytfs.size());
        for (size_t t = 0; t < mytfs.size(); t++) {
            coefs[t] = mycoeffs[t]->simplify(mydisjregs);
            isorientationdependent = isorientationdependent || coefs[t]->isvalueorientationdependent(mydisjregs);
            if (!coefs[t]->isharmonicone(mydisjregs))
                unsupported("a multiharmonic coefficient");
        }

        // Elements of all orientation groups, concatenated, with a variant index.
        std::vector<int> elems, variant, totalorients;
        std::shared_ptr<rawmesh> rm = universe::getrawmesh();
        const SelectorKey skey{rm.get(), rm->getmeshnumber(), isorientationdependent, mydisjregs};
        auto sit = tfphysreg == integrationphysreg ? g_selector_cache.find(skey) : g_selector_cache.end();
        if (sit != g_selector_cache.end() && sit->second.mesh.lock() == rm) {
            elems = sit->second.elems;
            variant = sit->second.variant;
            totalorients = sit->second.totalorients;
        } else {
            elementselector myselector;
            if (tfphysreg == integrationphysreg)
                myselector = elementselector(mydisjregs, isorientationdependent);
            else {
                std::vector<int> activeelems = gentools::getactiveelements(mydisjregs, isnodeintfphysreg);
                if (activeelems.size() > 0)
                    myselector = elementselector(mydisjregs, activeelems, isorientationdependent);
            }
            if (myselector.count() > 0)
                do {
                    std::vector<int> en = myselector.getelementnumbers();
                    int v = (int)totalorients.size();
                    totalorients.push_back(myselector.gettotalorientation());
                    elems.insert(elems.end(), en.begin(), en.end());
                    variant.insert(variant.end(), en.size(), v);
                } while (myselector.next());
            if (tfphysreg == integrationphysreg) {
                if (g_selector_cache.size() >= kSelectorEntries)
                    g_selector_cache.clear();
                g_selector_cache[skey] = SelectorEntry{rm, elems, variant, totalorients};
            }
        }
        if (elems.empty())
            continue;
        const int norient = (int)totalorients.size();
        const int nelem = (int)elems.size();

        // Form-function tables, deduplicated by (tf/dof, derivative, component).
        std::map<TableKey, int> tabindex;
        std::vector<std::vector<double>> tables;
        std::vector<int32_t> tablerows;
        auto table = [&](bool istf, int deriv, int comp) -> int {
            TableKey k{istf, deriv, comp};
            auto it = tabindex.find(k);
            if (it != tabindex.end())
                return it->second;
            hierarchicalformfunctioncontainer& c = istf ? tfval : dofval;
            const int order = istf ? tforder : doforder;
            std::vector<double> tab;
            int rows = -1;
            for (int o = 0; o < norient; o++) {
                densemat m = c.tomatrix(totalorients[o], order, deriv, comp);
                if (rows < 0) {
                    rows = m.countrows();
                    tab.resize((size_t)norient * rows * ngp);
                }
                std::copy(m.getvalues(), m.getvalues() + (size_t)rows * ngp, tab.begin() + (size_t)o * rows * ngp);
            }
            tables.push_back(std::move(tab));
            tablerows.push_back(rows);
            tabindex[k] = (int)tables.size() - 1;
            return (int)tables.size() - 1;
        };

        // Coefficient program and terms.
        Lowering low(mydisjregs, elemtype, elems, variant, totalorients, gpcoords);
        std::vector<int> tftab(mytfs.size()), doftab(mytfs.size(), -1), coefnode(mytfs.size()), dtorder(mytfs.size(), 0);
        for (size_t t = 0; t < mytfs.size(); t++) {
            tftab[t] = table(true, mytfs[t]->getkietaphiderivative(), mytfs[t]->getformfunctioncomponent());
            if (doffield != NULL) {
                doftab[t] = table(false, mydofs[t]->getkietaphiderivative(), mydofs[t]->getformfunctioncomponent());
                if (doffield->ismultiharmonic())
                    dtorder[t] = mydofs[t]->gettimederivative();
            }
        }
        low.field_table_base = (int)tables.size();
        for (size_t t = 0; t < mytfs.size(); t++) coefnode[t] = low.lower(coefs[t]);
        for (size_t k = 0; k < low.fieldtables.size(); k++) {
            tables.push_back(std::move(low.fieldtables[k]));
            tablerows.push_back(low.fieldtablerows[k]);
        }
        const int ntf = tablerows[tftab[0]];
        const int ndof = doffield != NULL ? tablerows[doftab[0]] : 1;

        // Harmonic folding (contribution.cpp:213-246): coefficient harmonic 1
        // times each dof harmonic gives scaled copies in the (tf, dof) blocks.
        // blocks[(tfharm, dofharm)] = per-term factors.
        std::map<std::pair<int, int>, std::vector<double>> blocks;
        for (size_t t = 0; t < mytfs.size(); t++) {
            for (int dh : dofharms) {
                std::vector<std::pair<int, double>> prods = harmonic::getproduct(1, dh, dtorder[t]);
                for (auto& pr : prods) {
                    if (!tffield->isharmonicincluded(pr.first))
                        continue;
                    auto& f = blocks[{pr.first, dh}];
                    if (f.empty())
                        f.assign(mytfs.size(), 0.0);
                    f[t] += pr.second;
                }
            }
        }
        // Units: blocks whose factor vectors are proportional share the
        // element matrices; each block becomes a destination with a multiplier.
        struct Unit {
            std::vector<double> scales;
            std::vector<std::pair<std::pair<int, int>, double>> dests;
        };
        std::vector<Unit> units;
        for (auto& b : blocks) {
            const std::vector<double>& f = b.second;
            size_t lead = 0;
            while (lead < f.size() && f[lead] == 0.0) lead++;
            if (lead == f.size())
                continue;
            std::vector<double> norm(f.size());
            for (size_t t = 0; t < f.size(); t++) norm[t] = f[t] / f[lead];
            bool placed = false;
            for (auto& u : units) {
                if (u.scales == norm) {
                    u.dests.push_back({b.first, f[lead]});
                    placed = true;
                    break;
                }
            }
            if (!placed)
                units.push_back(Unit{norm, {{b.first, f[lead]}}});
        }

        const int mesh_id = slgpu_adapter::ensure_mesh(elemtype);
        element curved(elemtype, universe::getrawmesh()->getelements()->getcurvatureorder());
        const int ncn = curved.countcurvednodes();
        lagrangeformfunction lag(elemtype, universe::getrawmesh()->getelements()->getcurvatureorder(), gpcoords);
        std::vector<double> lagrange((size_t)(1 + elemdim) * ncn * ngp);
        for (int d = 0; d <= elemdim; d++) {
            densemat m = lag.getderivative(d);
            std::copy(m.getvalues(), m.getvalues() + (size_t)ncn * ngp, lagrange.begin() + (size_t)d * ncn * ngp);
        }

        std::vector<slgpu_table> tabdesc(tables.size());
        for (size_t k = 0; k < tables.size(); k++) tabdesc[k] = slgpu_table{tablerows[k], tables[k].data()};
        std::vector<const double*> elemdataptr, fielddataptr;
        for (auto& v : low.elemdata) elemdataptr.push_back(v.data());
        for (auto& v : low.fielddata) fielddataptr.push_back(v.data());

        for (auto& u : units) {
            std::vector<slgpu_term> terms;
            for (size_t t = 0; t < mytfs.size(); t++) {
                if (u.scales[t] == 0.0)
                    continue;
                terms.push_back(slgpu_term{tftab[t], doftab[t], coefnode[t], 0, u.scales[t]});
            }
            std::vector<indexmat> addrkeep;
            std::vector<slgpu_dest> dests;
            for (auto& d : u.dests) {
                indexmat tfa = cached_addresses(mydofmanager, tffield->harmonic(d.first.first), tforder, elemtype, elems, tfphysreg);
                addrkeep.push_back(tfa);
                const int32_t* dofp = nullptr;
                if (doffield != NULL) {
                    indexmat dfa = cached_addresses(mydofmanager, doffield->harmonic(d.first.second), doforder, elemtype, elems, dofphysreg);
                    addrkeep.push_back(dfa);
                    dofp = dfa.getvalues();
                }
                dests.push_back(slgpu_dest{tfa.getvalues(), dofp, d.second});
            }
            slgpu_group g{};
            g.mesh = mesh_id;
            g.elemtype = elemtype;
            g.elemdim = elemdim;
            g.problemdim = meshdim;
            g.nelem = nelem;
            g.elems = elems.data();
            g.orient = variant.data();
            g.norient = norient;
            g.ngp = ngp;
            g.weights = weights.data();
            g.ncurvednodes = ncn;
            g.lagrange = lagrange.data();
            g.ntf = ntf;
            g.ndof = ndof;
            g.ntables = (int)tabdesc.size();
            g.tables = tabdesc.data();
            g.nnodes = (int)low.nodes.size();
            g.nodes = low.nodes.data();
            g.nconsts = (int)low.consts.size();
            g.consts = low.consts.data();
            g.nelemdata = (int)elemdataptr.size();
            g.elemdata = elemdataptr.data();
            g.nfielddata = (int)fielddataptr.size();
            g.fielddata = fielddataptr.data();
            g.fieldrows = low.fieldrows.data();
            g.nterms = (int)terms.size();
            g.terms = terms.data();
            g.ndests = (int)dests.size();
            g.dests = dests.data();

            if (doffield != NULL) {
                int handle = slgpu_adapter::matrix_handle(mymat.get(), ndofs);
                for (const indexmat& a : addrkeep) slgpu_adapter::keep_addresses(mymat.get(), a);
                slgpu_adapter::check(slgpu_matrix_add_group(ctx, handle, &g, nullptr), "slgpu_matrix_add_group");
            } else {
                // Right-hand side: b[addr] += -(element vectors), as
                // stiffnesses.minus() + rawvec::setvalues(..., "add"); only
                // the rows the group reaches are added.
                const int64_t cap = std::max<int64_t>(1, std::min<int64_t>(ndofs, (int64_t)ntf * nelem * (int64_t)dests.size()));
                std::vector<int32_t> rows((size_t)cap);
                std::vector<double> vals((size_t)cap);
                int64_t count = 0;
                int st = slgpu_rhs_assemble_rows(ctx, &g, ndofs, prec, rows.data(), vals.data(), cap, &count);
                if (st == SLGPU_E_NODEVICE && slgpu_adapter::record_only())
                    continue;  // recorded for inspection; nothing assembled
                slgpu_adapter::check(st, "slgpu_rhs_assemble_rows");
                if (count > 0) {
                    indexmat ri((long long)count, 1);
                    densemat vi((long long)count, 1);
                    std::copy(rows.begin(), rows.begin() + count, ri.getvalues());
                    std::copy(vals.begin(), vals.begin() + count, vi.getvalues());
                    myvec->setvalues(ri, vi, "add");
                }
            }
        }
    }
}

namespace slgpu_adapter {
void clear_address_cache(void) { g_address_cache.clear(); }
}  // namespace slgpu_adapter
