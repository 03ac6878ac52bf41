"""Reader of the reference's ``.nrg`` system files, feeding ``System``.

Mirrors ``tools::ReadNrg`` / ``ReadSystem`` / ``ReadMolecule`` /
``ReadMonomers`` (io_tools/read_nrg.cpp:43-290): a file holds one or more
systems::

    SYSTEM <label>
    MOLECULE <label>
    MONOMER <id>
    <atom> <x> <y> <z>
    ...
    ENDMON
    ENDMOL
    ...
    ENDSYS

Keywords are case-insensitive, monomer ids are lower-cased, atom names are
kept as written.  Reading stops at the end of the file or at an empty line
after a system.  Errors name the line, like the reference's CUException
texts.  Kept as in the reference: within one MOLECULE, a second MONOMER
line's id is not read again -- every monomer of a molecule carries the id of
its first MONOMER line (read_nrg.cpp:206-216 read the id once, the loop only
re-reads the keyword).
"""
from .system import CUException, System


class NrgSystem:
    """One system of an .nrg file: monomer ids, atom names and coordinates in
    input order, molecules as lists of monomer indices."""

    def __init__(self, label):
        self.label = label
        self.ids = []
        self.atoms = []
        self.xyz = []
        self.molecules = []

    def coordinates(self):
        out = []
        for x in self.xyz:
            out.extend(x)
        return out

    def to_system(self, json_text=None, device=0, context=None):
        """The initialised System (System::Initialize as ReadSystem does, then
        SetUpFromJson when a configuration is given)."""
        s = System(device, context)
        for mid, names, x in zip(self.ids, self.atoms, self.xyz):
            s.AddMonomer(x, names, mid)
        for m in self.molecules:
            s.AddMolecule(m)
        s.Initialize()
        if json_text is not None:
            s.SetUpFromJson(json_text)
        return s


def _lines(text):
    for n, line in enumerate(text.splitlines(), 1):
        yield n, line


def parse_nrg(text):
    """All systems of an .nrg text (list of NrgSystem)."""
    lines = list(_lines(text))
    pos = 0
    systems = []

    def next_line():
        nonlocal pos
        if pos >= len(lines):
            raise CUException("Unexpected end of the NRG file after line %d" % (lines[-1][0] if lines else 0))
        n, line = lines[pos]
        pos += 1
        return n, line

    def first_word(line):
        w = line.split()
        return w[0].lower() if w else None

    while True:
        n, line = next_line()
        w = line.split()
        if not w:
            raise CUException("Unexpected text at line %d of the NRG file:\n%s" % (n, line))
        if w[0].lower() != "system":
            raise CUException("Expected SYSTEM keyword in line  %d of the NRG file.\nFound %s" % (n, line))
        sys_ = NrgSystem(" ".join(w[1:]))
        mon_count = 0
        word = "system"
        while word != "endsys":
            # ReadMolecule
            n, line = next_line()
            if first_word(line) is None:
                raise CUException("Unexpected text at line %d of the NRG file:\n%s" % (n, line))
            if first_word(line) != "molecule":
                raise CUException("Expected MOLECULE keyword in line  %d of the NRG file.\nFound %s" % (n, line))
            # ReadMonomers
            n, line = next_line()
            w = line.split()
            if not w:
                raise CUException("Unexpected text at line %d of the NRG file:\n%s" % (n, line))
            if w[0].lower() != "monomer":
                raise CUException("Expected MONOMER keyword in line  %d of the NRG file.\nFound %s" % (n, line))
            mon_name = w[1].lower() if len(w) > 1 else ""
            word = "monomer"
            molec = []
            while word != "endmol":
                if word != "monomer" or not mon_name:
                    raise CUException("Expected MONOMER keyword in line  %d of the NRG file, along with the "
                                      "monomer id.\nFound %s" % (n, line))
                names, xyz = [], []
                n, line = next_line()
                word = first_word(line)
                while word != "endmon":
                    t = line.split()
                    if len(t) < 2:
                        raise CUException("Expected coordinates or ENDMON in line  %d of the NRG file.\n"
                                          "Found: %s" % (n, line))
                    try:
                        x, y, z = (float(v) for v in t[1:4])
                    except ValueError:
                        raise CUException("Expected numerical coordinates in line  %d of the NRG file.\n"
                                          "Found: %s" % (n, line))
                    names.append(t[0])
                    xyz.extend((x, y, z))
                    n, line = next_line()
                    word = first_word(line)
                sys_.ids.append(mon_name)
                sys_.atoms.append(names)
                sys_.xyz.append(xyz)
                molec.append(mon_count)
                mon_count += 1
                n, line = next_line()
                word = first_word(line)
            sys_.molecules.append(molec)
            # after ENDMOL: the next line is ENDSYS or another MOLECULE
            n, line = next_line()
            word = first_word(line)
            if word == "molecule":
                pos -= 1
        systems.append(sys_)
        if pos >= len(lines) or not lines[pos][1].strip():
            break
    return systems


def read_nrg(path):
    """tools::ReadNrg: all systems of an .nrg file."""
    try:
        text = open(path).read()
    except OSError:
        raise CUException("Could not open NRG file %s for reading." % path)
    return parse_nrg(text)


def format_nrg(systems):
    """.nrg text of systems (NrgSystem), readable by read_nrg and by the
    reference's ReadNrg."""
    out = []
    for s in systems:
        out.append("SYSTEM %s" % (s.label or "0"))
        for mi, molec in enumerate(s.molecules):
            out.append("MOLECULE %d" % mi)
            for m in molec:
                out.append("MONOMER %s" % s.ids[m])
                x = s.xyz[m]
                for a, name in enumerate(s.atoms[m]):
                    out.append("%s %.17g %.17g %.17g" % (name, x[3 * a], x[3 * a + 1], x[3 * a + 2]))
                out.append("ENDMON")
            out.append("ENDMOL")
        out.append("ENDSYS")
    return "\n".join(out) + "\n"
