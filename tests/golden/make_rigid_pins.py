"""Extracts the values the reference's own rigid-body tests pin into JSON
fixtures: tests/block-sliding.py:64-80 (position x and velocity v_x of the
block at given callback indices, 1e-3 relative tolerance) into
block_sliding_ref.json, tests/projectile.py:47-50 (the x distance in
inches at the end, 0.5% relative tolerance) into projectile_ref.json,
tests/math-pendulum.py:31-35 (the period from the horizontal, 1%) into
math_pendulum_ref.json, tests/pinned-bar.py:38-42 (the angular velocity about
y when the mass centre passes x = 0, 1%) into pinned_bar_ref.json and
tests/double-pendulum.py:103-107 (total energy at given step indices, 1e-3
relative to max(1, value)) into double_pendulum_ref.json. Run with
the environment variable REFERENCE set to the reference source tree; the
tests read only the JSON."""
import ast
import json
import os
import re
import sys

REFERENCE = os.environ.get('REFERENCE')


def main():
    if not REFERENCE or not os.path.isdir(REFERENCE):
        sys.exit('set REFERENCE to the reference source tree')
    src = open(os.path.join(REFERENCE, 'tests', 'block-sliding.py')).read()
    m = re.search(r'REF\s*=\s*(\[[^\]]*\])', src)  # the test is Python 2: read the list literal alone
    if not m:
        sys.exit('REF list not found')
    values = ast.literal_eval(m.group(1))
    out = dict(source='tests/block-sliding.py of the reference (REF list)', tolerance=1e-3,
               step=1e-3, stop=10.0, friction=0.8, gravity=9.81,
               pins=[dict(quantity='x' if k == 0 else 'vx', index=int(i), value=float(v)) for k, i, v in values])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'block_sliding_ref.json')
    with open(path, 'w') as f:
        json.dump(out, f, indent=1)
    print(path, len(values), 'pins')
    src = open(os.path.join(REFERENCE, 'tests', 'projectile.py')).read()
    exact = float(re.search(r'exact\s*=\s*([0-9.eE+-]+)', src).group(1))
    tol = float(re.search(r'if \(error < ([0-9.eE+-]+)\)', src).group(1))
    out = dict(source='tests/projectile.py of the reference (exact, error bound)', quantity='x distance [in]',
               value=exact, tolerance=tol)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'projectile_ref.json')
    with open(path, 'w') as f:
        json.dump(out, f, indent=1)
    print(path, exact, tol)
    here = os.path.dirname(os.path.abspath(__file__))
    for test, out_name, quantity in (('math-pendulum.py', 'math_pendulum_ref.json', 'period [s]'),
                                     ('pinned-bar.py', 'pinned_bar_ref.json', 'angular velocity about y [rad/s]')):
        src = open(os.path.join(REFERENCE, 'tests', test)).read()
        exact = float(re.search(r'exact\s*=\s*([0-9.eE+-]+)', src).group(1))
        tol = float(re.search(r'if \(error < ([0-9.eE+-]+)\)', src).group(1))
        out = dict(source='tests/%s of the reference (exact, error bound)' % test, quantity=quantity, value=exact,
                   tolerance=tol)
        with open(os.path.join(here, out_name), 'w') as f:
            json.dump(out, f, indent=1)
        print(out_name, exact, tol)
    src = open(os.path.join(REFERENCE, 'tests', 'double-pendulum.py')).read()
    m = re.search(r'REF\s*=\s*(\[[^\]]*\])', src)
    tol = float(re.search(r'if error > ([0-9.eE+-]+)', src).group(1))
    values = ast.literal_eval(m.group(1))
    out = dict(source='tests/double-pendulum.py of the reference (REF list)', quantity='total energy [J]',
               tolerance=tol, pins=[dict(index=int(i), value=float(v)) for i, v in values])
    with open(os.path.join(here, 'double_pendulum_ref.json'), 'w') as f:
        json.dump(out, f, indent=1)
    print('double_pendulum_ref.json', len(values), tol)


if __name__ == '__main__':
    main()
