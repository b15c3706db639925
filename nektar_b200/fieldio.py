"""Nektar++ .fld output in the XML format (FieldIOXml), so that a solution of
the B200 path opens in the reference's post-processing tools.

Layout, as FieldIOXml::v_Write (LibUtilities/BasicUtils/FieldIOXml.cpp:
83-346) and SetUpFieldMetaData (:652-716) produce it for one process: `out.fld`
is a directory holding

* `Info.xml`: `<NEKTAR><Metadata><Provenance>...</Provenance>...</Metadata>
  <Partition FileName="P0000000.fld">ids</Partition></NEKTAR>`
  (WriteMultiFldFileIDs, :372-403; FieldIO::AddInfoTag, FieldIO.cpp:339-382);
* `P0000000.fld`: `<NEKTAR>` with the same metadata and one `<ELEMENTS>`
  block per field definition (shape, basis, orders): attributes FIELDS,
  SHAPE, BASIS, NUMMODESPERDIR ("UNIORDER:6,6,6"), ID (a sequence string),
  COMPRESSED ("B64Z-LittleEndian"), BITSIZE ("64"); the text is the field
  data, every field's coefficients element by element in the element's own
  coefficient order, as little-endian doubles, zlib-compressed and base64
  encoded (CompressData::ZlibEncodeToBase64Str).
"""
import base64
import datetime
import os
import shutil
import socket
import xml.etree.ElementTree as ET
import zlib

import numpy as np

SHAPE_NAMES = {"hex": "Hexahedron", "prism": "Prism", "tet": "Tetrahedron"}
BASIS_NAMES = {"hex": ("Modified_A", "Modified_A", "Modified_A"),
               "prism": ("Modified_A", "Modified_A", "Modified_B"),
               "tet": ("Modified_A", "Modified_B", "Modified_C")}
VERSION = "5.10.0"


def seq_string(ids):
    """[0, 1, 2, 5] -> '0-2,5' (ParseUtils::GenerateSeqString)."""
    ids = list(ids)
    out, i = [], 0
    while i < len(ids):
        j = i
        while j + 1 < len(ids) and ids[j + 1] == ids[j] + 1:
            j += 1
        out.append(str(ids[i]) if i == j else "%d-%d" % (ids[i], ids[j]))
        i = j + 1
    return ",".join(out)


def _metadata(root, extra=None):
    md = ET.SubElement(root, "Metadata")
    prov = ET.SubElement(md, "Provenance")
    stamp = datetime.datetime.now().strftime("%d-%b-%Y %H:%M:%S")
    for k, v in sorted({"NektarVersion": VERSION, "Timestamp": stamp,
                        "Hostname": socket.gethostname()}.items()):
        ET.SubElement(prov, k).text = v
    for k, v in (extra or {}).items():
        ET.SubElement(md, k).text = str(v)


def encode(data):
    """B64Z-LittleEndian encoding of a float64 array."""
    raw = np.ascontiguousarray(data, dtype="<f8").tobytes()
    return base64.b64encode(zlib.compress(raw)).decode("ascii")


def decode(text):
    return np.frombuffer(zlib.decompress(base64.b64decode(text.strip())), dtype="<f8").copy()


def _write_xml(root, path):
    ET.indent(root)
    with open(path, "wb") as fh:
        fh.write(b'<?xml version="1.0" encoding="utf-8" ?>\n')
        fh.write(ET.tostring(root))


def write_fld(path, mesh, fields, metadata=None):
    """Write fields {name: local coefficients (the mesh's concatenated local
    vector)} of a session mesh as the directory `path`: one ELEMENTS block
    per collection (shape and order), as GetFieldDefinitions groups them."""
    names = list(fields)
    if os.path.isdir(path):
        shutil.rmtree(path)
    elif os.path.exists(path):
        os.remove(path)
    os.makedirs(path)
    root = ET.Element("NEKTAR")
    _metadata(root, metadata)
    all_ids = []
    for ci, col in enumerate(mesh.collections):
        lo, hi = int(mesh.offsets[ci]), int(mesh.offsets[ci + 1])
        # field by field, element by element (ExpList::AppendFieldData per field)
        data = np.concatenate([np.asarray(fields[n], dtype=np.float64).reshape(-1)[lo:hi]
                               for n in names])
        ids = list(col.elem_ids)  # in the order their data follows
        all_ids += ids
        el = ET.SubElement(root, "ELEMENTS")
        el.set("FIELDS", ",".join(names))
        el.set("SHAPE", SHAPE_NAMES[col.shape])
        el.set("BASIS", ",".join(BASIS_NAMES[col.shape]))
        el.set("NUMMODESPERDIR", "UNIORDER:%d,%d,%d" % (col.nm, col.nm, col.nm))
        el.set("ID", seq_string(ids))
        el.set("COMPRESSED", "B64Z-LittleEndian")
        el.set("BITSIZE", "64")
        el.text = encode(data)
    _write_xml(root, os.path.join(path, "P0000000.fld"))
    info = ET.Element("NEKTAR")
    _metadata(info, metadata)
    part = ET.SubElement(info, "Partition")
    part.set("FileName", "P0000000.fld")
    part.text = seq_string(all_ids)
    _write_xml(info, os.path.join(path, "Info.xml"))


def read_fld(path):
    """(definitions, data) of a .fld directory written as above: one dict per
    ELEMENTS block with its attributes, element ids and the decoded data."""
    files = [path]
    if os.path.isdir(path):
        info = ET.parse(os.path.join(path, "Info.xml")).getroot()
        files = [os.path.join(path, p.get("FileName")) for p in info.findall("Partition")]
    out = []
    from .session import parse_id_list
    for f in files:
        for el in ET.parse(f).getroot().findall("ELEMENTS"):
            d = dict(el.attrib)
            d["ids"] = parse_id_list(d["ID"])
            d["fields"] = d["FIELDS"].split(",")
            d["data"] = decode(el.text)
            out.append(d)
    return out
